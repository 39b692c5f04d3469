// DG kernels: face traces (restriction), admissibility, frozen HLL speeds and CFL rate,
// the weak residual R(u), the linearisation caches (u, v, H only), the matrix-free J·v and
// the dense diagonal block assembly.  One thread team per cell; N = k+1 is a template constant.
#pragma once
#include "dgh_common.cuh"

namespace dgh {

template <int N> struct Team {
    static constexpr int P = N * N;
    static constexpr int TPC = ((P + 31) / 32) * 32;          // threads per cell
    static constexpr int CPB = TPC >= 128 ? 1 : 128 / TPC;    // cells per CTA
    static constexpr int THREADS = TPC * CPB;
};

// ---- face restriction (discretization.cpp:50-60,73-87) -------------------------------------
// traces[(cell*4 + side)*N*4 + q*4 + v] = sum_i e_side[i] u[v][face_node(side,q,i)]
// Optionally checks admissibility (discretization.cpp:211-233): every nodal value finite, and
// density and pressure above 1e-13 at the nodes and the four face restrictions.
// (The kernel bodies below take their block index bx explicitly, so the batched kernels of a
// lockstep batch run the same arithmetic per member.)
template <int N, bool CHECK>
__device__ __forceinline__ void face_trace_body(int bx, const double *__restrict__ u, double *__restrict__ traces,
                                                const Basis1D &b, const Grid &g, int *ok) {
    using T = Team<N>;
    __shared__ double su[T::CPB][NVAR * T::P];
    const int sub = threadIdx.x / T::TPC, lt = threadIdx.x % T::TPC;
    const int cell = bx * T::CPB + sub;
    const bool active = cell < g.cells;
    const double *uc = u + (size_t)cell * NVAR * T::P;
    if (active)
        for (int k = lt; k < NVAR * T::P; k += T::TPC) su[sub][k] = uc[k];
    __syncthreads();
    if (!active) return;
    bool good = true;
    if (CHECK)
        for (int node = lt; node < T::P; node += T::TPC) {
            double s[4] = {su[sub][node], su[sub][T::P + node], su[sub][2 * T::P + node], su[sub][3 * T::P + node]};
            const bool finite = isfinite(s[0]) && isfinite(s[1]) && isfinite(s[2]) && isfinite(s[3]);
            if (!finite || s[0] <= 1e-13 || !(pressure(g.gamma, s) > 1e-13)) good = false;
        }
    double *tc = traces + (size_t)cell * NFACES * N * NVAR;
    for (int k = lt; k < NFACES * N; k += T::TPC) {
        const int side = k / N, q = k % N;
        const double *e = side % 2 ? b.eR : b.eL;
        double s[4];
#pragma unroll
        for (int v = 0; v < NVAR; ++v) {
            double acc = 0;
#pragma unroll
            for (int i = 0; i < N; ++i) acc = rfma(e[i], su[sub][v * T::P + face_node(N, side, q, i)], acc);
            s[v] = acc;
            tc[k * NVAR + v] = acc;
        }
        if (CHECK) {
            const bool finite = isfinite(s[0]) && isfinite(s[1]) && isfinite(s[2]) && isfinite(s[3]);
            if (!finite || s[0] <= 1e-13 || !(pressure(g.gamma, s) > 1e-13)) good = false;
        }
    }
    if (CHECK && !good) atomicExch(ok, 0);
}
template <int N, bool CHECK>
__global__ void __launch_bounds__(Team<N>::THREADS)
k_face_trace(const double *__restrict__ u, double *__restrict__ traces, Basis1D b, Grid g, int *ok) {
    face_trace_body<N, CHECK>(blockIdx.x, u, traces, b, g, ok);
}

// ---- frozen HLL speeds (discretization.cpp:163-177) -----------------------------------------
// speeds[2*(face*N+q)] = a, [+1] = b
template <int N>
__global__ void k_speeds(const double *__restrict__ traces, double *__restrict__ speeds, Grid g, double safety,
                         int *status) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 2 * g.cells * N) return;
    const int face = idx / N, q = idx % N;
    const int axis = face >= g.cells, cell = face - axis * g.cells;
    const int side = 2 * axis + 1, next = neighbor(g, cell, side);
    const double *L = traces + ((size_t)cell * NFACES + side) * N * NVAR + q * NVAR;
    const double *R = traces + ((size_t)next * NFACES + side - 1) * N * NVAR + q * NVAR;
    double l[4] = {L[0], L[1], L[2], L[3]}, r[4] = {R[0], R[1], R[2], R[3]};
    double a, bb;
    if (!einfeldt(g.gamma, l, r, safety, axis, a, bb)) atomicOr(status, ST_FROZEN_FACE);
    speeds[2 * idx] = a;
    speeds[2 * idx + 1] = bb;
}

// ---- CFL rate per cell (discretization.cpp:178-195); block partial maxima -------------------
template <int N>
__global__ void __launch_bounds__(Team<N>::THREADS)
k_rate(const double *__restrict__ u, const double *__restrict__ speeds, Grid g, double *__restrict__ partial,
       int *status, int first, int last) {
    using T = Team<N>;
    __shared__ double sa[T::THREADS], sb[T::THREADS];
    const int sub = threadIdx.x / T::TPC, lt = threadIdx.x % T::TPC;
    const int cell = first + blockIdx.x * T::CPB + sub;  // cells [first, last)
    double ax = 0, ay = 0;
    if (cell < last) {
        for (int k = lt; k < NFACES * N; k += T::TPC) {
            const int side = k / N, q = k % N;
            const int face = face_of(g, cell, side);
            const double s = fmax(speeds[2 * (face * N + q)], speeds[2 * (face * N + q) + 1]);
            if (side < 2) ax = fmax(ax, s); else ay = fmax(ay, s);
        }
        const double *uc = u + (size_t)cell * NVAR * T::P;
        for (int node = lt; node < T::P; node += T::TPC) {
            double s[4] = {uc[node], uc[T::P + node], uc[2 * T::P + node], uc[3 * T::P + node]};
            const Prim p = primitive(g.gamma, s);
            if (!(s[0] > 0 && p.p > 0)) atomicOr(status, ST_CFL_VOLUME);
            const double c = sqrt(g.gamma * p.p * p.ir);
            ax = fmax(ax, fabs(p.vx) + c);
            ay = fmax(ay, fabs(p.vy) + c);
        }
    }
    sa[threadIdx.x] = ax;
    sb[threadIdx.x] = ay;
    __syncthreads();
    if (threadIdx.x == 0) {
        double best = 0;
        for (int c = 0; c < T::CPB; ++c) {
            if (first + blockIdx.x * T::CPB + c >= last) break;
            double mx = 0, my = 0;
            for (int t = 0; t < T::TPC; ++t) {
                mx = fmax(mx, sa[c * T::TPC + t]);
                my = fmax(my, sb[c * T::TPC + t]);
            }
            best = fmax(best, mx / g.hx + my / g.hy);
        }
        partial[blockIdx.x] = best;
    }
}

// ---- weak residual (discretization.cpp:111-140, tensor_product.cpp:41-56) --------------------
// r = M (u - old)/tau - (hy/2)(Dw)^T Fx W - (hx/2) W Fy Dw + sum_sides (+/-) e_s HLL(u_L, u_R)
template <int N>
__global__ void __launch_bounds__(Team<N>::THREADS)
k_residual(const double *__restrict__ u, const double *__restrict__ old, const double *__restrict__ traces,
           const double *__restrict__ speeds, double *__restrict__ r, Basis1D b, Grid g, double inv_step,
           int volterm = 1) {
    using T = Team<N>;
    __shared__ double fx[T::CPB][NVAR * T::P], fy[T::CPB][NVAR * T::P];
    __shared__ double ff[T::CPB][NFACES * N * NVAR];
    const int sub = threadIdx.x / T::TPC, lt = threadIdx.x % T::TPC;
    const int cell = blockIdx.x * T::CPB + sub;
    const bool active = cell < g.cells;
    const size_t base = (size_t)cell * NVAR * T::P;
    double uu[4] = {0, 0, 0, 0};
    if (active && lt < T::P) {
#pragma unroll
        for (int v = 0; v < NVAR; ++v) uu[v] = u[base + v * T::P + lt];
        double a[4], c[4];
        flux(g.gamma, uu, 0, a);
        flux(g.gamma, uu, 1, c);
#pragma unroll
        for (int v = 0; v < NVAR; ++v) {
            fx[sub][v * T::P + lt] = a[v];
            fy[sub][v * T::P + lt] = c[v];
        }
    }
    if (active)
        for (int k = lt; k < NFACES * N; k += T::TPC) {
            const int side = k / N, q = k % N, axis = side / 2;
            const int nb = neighbor(g, cell, side), face = face_of(g, cell, side);
            const double *own = traces + ((size_t)cell * NFACES + side) * N * NVAR + q * NVAR;
            const double *oth = traces + ((size_t)nb * NFACES + (side ^ 1)) * N * NVAR + q * NVAR;
            double L[4], R[4];
#pragma unroll
            for (int v = 0; v < NVAR; ++v) {
                L[v] = side % 2 ? own[v] : oth[v];
                R[v] = side % 2 ? oth[v] : own[v];
            }
            const double sa = speeds[2 * (face * N + q)], sb = speeds[2 * (face * N + q) + 1];
            double fl[4], fr[4];
            flux(g.gamma, L, axis, fl);
            flux(g.gamma, R, axis, fr);
            const double scale = face_weight(g, b, face, q) / (sa + sb);
            const double sign = side % 2 ? 1. : -1.;
#pragma unroll
            for (int v = 0; v < NVAR; ++v)
                ff[sub][k * NVAR + v] = sign * (scale * (sb * fl[v] + sa * fr[v] + sa * sb * (L[v] - R[v])));
        }
    __syncthreads();
    if (!active || lt >= T::P) return;
    const int ix = lt % N, iy = lt / N;
    const double mass = .25 * g.hx * g.hy * b.w[ix] * b.w[iy];
    const double sx = .5 * g.hy, sy = .5 * g.hx;
#pragma unroll
    for (int v = 0; v < NVAR; ++v) {
        double wx = 0, wy = 0;
#pragma unroll
        for (int q = 0; q < N; ++q) {
            wx += b.dw[q * N + ix] * fx[sub][v * T::P + q + N * iy];
            wy += fy[sub][v * T::P + ix + N * q] * b.dw[q * N + iy];
        }
        double val = mass * (uu[v] - old[base + v * T::P + lt]) * inv_step;
        if (N > 1 && volterm) val -= sx * b.w[iy] * wx + sy * b.w[ix] * wy;
        val += b.eL[ix] * ff[sub][(0 * N + iy) * NVAR + v] + b.eR[ix] * ff[sub][(1 * N + iy) * NVAR + v] +
               b.eL[iy] * ff[sub][(2 * N + ix) * NVAR + v] + b.eR[iy] * ff[sub][(3 * N + ix) * NVAR + v];
        r[base + v * T::P + lt] = val;
    }
}

// ---- linearisation caches (volume_jacobian.cpp:30-42, face_jacobian.cpp:16-37) -------------
// vol[(cell*P + node)*3 + {0,1,2}] = u, v, H
template <int N>
__global__ void k_volume_cache(const double *__restrict__ u, double *__restrict__ vol, Grid g) {
    constexpr int P = N * N;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)g.cells * P) return;
    const int cell = idx / P, node = idx % P;
    const double *uc = u + (size_t)cell * NVAR * P;
    double s[4] = {uc[node], uc[P + node], uc[2 * P + node], uc[3 * P + node]};
    const Prim p = primitive(g.gamma, s);
    vol[idx * 3] = p.vx;
    vol[idx * 3 + 1] = p.vy;
    vol[idx * 3 + 2] = p.H;
}
// fcache[(face*N + q)*8 + k]: k 0..2 left (u,v,H), 3..5 right (u,v,H), 6 blend_l, 7 blend_r;
// penalty = w a b/(a+b) is recomputed from the speeds where needed.
template <int N>
__global__ void k_face_cache(const double *__restrict__ traces, const double *__restrict__ speeds,
                             double *__restrict__ fcache, Basis1D b, Grid g) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 2 * g.cells * N) return;
    const int face = idx / N, q = idx % N;
    const int axis = face >= g.cells, cell = face - axis * g.cells;
    const int side = 2 * axis + 1, next = neighbor(g, cell, side);
    const double *L = traces + ((size_t)cell * NFACES + side) * N * NVAR + q * NVAR;
    const double *R = traces + ((size_t)next * NFACES + side - 1) * N * NVAR + q * NVAR;
    double l[4] = {L[0], L[1], L[2], L[3]}, r[4] = {R[0], R[1], R[2], R[3]};
    const Prim pl = primitive(g.gamma, l), pr = primitive(g.gamma, r);
    const double a = speeds[2 * idx], bb = speeds[2 * idx + 1], w = face_weight(g, b, face, q);
    double *c = fcache + (size_t)idx * 8;
    c[0] = pl.vx; c[1] = pl.vy; c[2] = pl.H;
    c[3] = pr.vx; c[4] = pr.vy; c[5] = pr.H;
    c[6] = w * bb / (a + bb);
    c[7] = w * a / (a + bb);
}

// normal_action (dgh_common.cuh) with every product and sum explicitly rounded, for the J·v
// body shared by the single-problem and the lockstep kernels (same bits in both).
__device__ __forceinline__ void normal_action_rn(double gamma, double u, double v, double H, const double d[4], int axis,
                                                 double out[4]) {
    const double dr = d[0], dx = d[1], dy = d[2], de = d[3];
    const double q2 = rfma(u, u, rmul(v, v));
    double t = rfma(-u, dx, de);
    t = rfma(-v, dy, t);
    t = rfma(rmul(.5, q2), dr, t);
    const double dp = rmul(rsub(gamma, 1.), t);
    const double uv = rmul(u, v);
    if (axis == 0) {
        out[0] = dx;
        out[1] = rfma(rmul(2., u), dx, rfma(-rmul(u, u), dr, dp));
        out[2] = rfma(u, dy, rfma(v, dx, -rmul(uv, dr)));
        out[3] = rfma(H, rfma(-u, dr, dx), rmul(u, radd(de, dp)));
    } else {
        out[0] = dy;
        out[1] = rfma(u, dy, rfma(v, dx, -rmul(uv, dr)));
        out[2] = rfma(rmul(2., v), dy, rfma(-rmul(v, v), dr, dp));
        out[3] = rfma(H, rfma(-v, dr, dy), rmul(v, radd(de, dp)));
    }
}

// ---- matrix-free J·v (volume_jacobian.cpp:59-71 + dg_operator.cpp:10-21) ---------------------
// Needs the face traces of the direction d (k_face_trace on d).
template <int N>
__device__ __forceinline__ void dg_apply_body(int bx, const double *__restrict__ d, const double *__restrict__ dtr,
                                              const double *__restrict__ vol, const double *__restrict__ fcache,
                                              const double *__restrict__ speeds, double *__restrict__ out,
                                              const Basis1D *__restrict__ bp, const Grid &g, double inv_step,
                                              int volterm) {
    // the basis tables are indexed per thread: read them through L1 from a device copy rather
    // than from the kernel's parameter bank, where lane-varying indices serialise
    const Basis1D &b = *bp;
    using T = Team<N>;
    __shared__ double fx[T::CPB][NVAR * T::P], fy[T::CPB][NVAR * T::P];
    __shared__ double ff[T::CPB][NFACES * N * NVAR];
    const int sub = threadIdx.x / T::TPC, lt = threadIdx.x % T::TPC;
    const int cell = bx * T::CPB + sub;
    const bool active = cell < g.cells;
    const size_t base = (size_t)cell * NVAR * T::P;
    double dd[4] = {0, 0, 0, 0};
    if (active && lt < T::P) {
#pragma unroll
        for (int v = 0; v < NVAR; ++v) dd[v] = d[base + v * T::P + lt];
        const double *c = vol + ((size_t)cell * T::P + lt) * 3;
        double a[4], e[4];
        normal_action_rn(g.gamma, c[0], c[1], c[2], dd, 0, a);
        normal_action_rn(g.gamma, c[0], c[1], c[2], dd, 1, e);
#pragma unroll
        for (int v = 0; v < NVAR; ++v) {
            fx[sub][v * T::P + lt] = a[v];
            fy[sub][v * T::P + lt] = e[v];
        }
    }
    if (active)
        for (int k = lt; k < NFACES * N; k += T::TPC) {
            const int side = k / N, q = k % N, axis = side / 2;
            const int nb = neighbor(g, cell, side), face = face_of(g, cell, side);
            const double *own = dtr + ((size_t)cell * NFACES + side) * N * NVAR + q * NVAR;
            const double *oth = dtr + ((size_t)nb * NFACES + (side ^ 1)) * N * NVAR + q * NVAR;
            double L[4], R[4];
#pragma unroll
            for (int v = 0; v < NVAR; ++v) {
                L[v] = side % 2 ? own[v] : oth[v];
                R[v] = side % 2 ? oth[v] : own[v];
            }
            const double *c = fcache + ((size_t)face * N + q) * 8;
            double al[4], ar[4];
            normal_action_rn(g.gamma, c[0], c[1], c[2], L, axis, al);
            normal_action_rn(g.gamma, c[3], c[4], c[5], R, axis, ar);
            const double sa = speeds[2 * (face * N + q)], sb = speeds[2 * (face * N + q) + 1];
            const double pen = rmul(rmul(face_weight(g, b, face, q), sa), sb) / radd(sa, sb);
            const double sign = side % 2 ? 1. : -1.;
#pragma unroll
            for (int v = 0; v < NVAR; ++v)
                ff[sub][k * NVAR + v] = rmul(sign, rfma(c[6], al[v], rfma(c[7], ar[v], rmul(pen, rsub(L[v], R[v])))));
        }
    __syncthreads();
    if (!active || lt >= T::P) return;
    const int ix = lt % N, iy = lt / N;
    const double mass = rmul(rmul(rmul(rmul(.25, g.hx), g.hy), b.w[ix]), b.w[iy]);
    const double sxw = rmul(rmul(.5, g.hy), b.w[iy]), syw = rmul(rmul(.5, g.hx), b.w[ix]);
#pragma unroll
    for (int v = 0; v < NVAR; ++v) {
        double wx = 0, wy = 0;
#pragma unroll
        for (int q = 0; q < N; ++q) {
            wx = rfma(b.dw[q * N + ix], fx[sub][v * T::P + q + N * iy], wx);
            wy = rfma(fy[sub][v * T::P + ix + N * q], b.dw[q * N + iy], wy);
        }
        double val = rmul(rmul(mass, dd[v]), inv_step);
        if (N > 1 && volterm) val = rsub(val, rfma(sxw, wx, rmul(syw, wy)));
        const double lift = rfma(b.eL[ix], ff[sub][(0 * N + iy) * NVAR + v],
                                 rfma(b.eR[ix], ff[sub][(1 * N + iy) * NVAR + v],
                                      rfma(b.eL[iy], ff[sub][(2 * N + ix) * NVAR + v],
                                           rmul(b.eR[iy], ff[sub][(3 * N + ix) * NVAR + v]))));
        out[base + v * T::P + lt] = radd(val, lift);
    }
}
template <int N>
__global__ void __launch_bounds__(Team<N>::THREADS, 65536 / (Team<N>::THREADS * 72))
k_dg_apply(const double *__restrict__ d, const double *__restrict__ dtr, const double *__restrict__ vol,
           const double *__restrict__ fcache, const double *__restrict__ speeds, double *__restrict__ out,
           const Basis1D *__restrict__ bp, Grid g, double inv_step, int volterm = 1) {
    dg_apply_body<N>(blockIdx.x, d, dtr, vol, fcache, speeds, out, bp, g, inv_step, volterm);
}

// ---- adjoint J^T w (the transpose of k_dg_apply, same frozen speeds and caches) -------------
// Volume: for node (a, b), gx = sum_i dw[a n + i] w(i, b) and gy = sum_j dw[b n + j] w(a, j);
// (J^T w)(a, b) = M w / tau - (hy/2) w_b Ax^T gx - (hx/2) w_a Ay^T gy.  Faces: with the jump
// z = E_right-side w_L - E_left-side w_R of the two cells sharing a face, the left cell receives
// lift((blend_l A_L + pen I)^T z) and the right cell lift((blend_r A_R - pen I)^T z).
// Needs the face traces of w (k_face_trace on w).  volterm = 0 leaves out the collocated volume
// term (the over-integrated rule adds its own, k_vol_apply_q_t).
template <int N>
__global__ void __launch_bounds__(Team<N>::THREADS)
k_dg_apply_t(const double *__restrict__ w, const double *__restrict__ wtr, const double *__restrict__ vol,
             const double *__restrict__ fcache, const double *__restrict__ speeds, double *__restrict__ out,
             Basis1D b, Grid g, double inv_step, int volterm = 1) {
    using T = Team<N>;
    __shared__ double ws[T::CPB][NVAR * T::P];
    __shared__ double ff[T::CPB][NFACES * N * NVAR];
    const int sub = threadIdx.x / T::TPC, lt = threadIdx.x % T::TPC;
    const int cell = blockIdx.x * T::CPB + sub;
    const bool active = cell < g.cells;
    const size_t base = (size_t)cell * NVAR * T::P;
    if (active)
        for (int k = lt; k < NVAR * T::P; k += T::TPC) ws[sub][k] = w[base + k];
    if (active)
        for (int k = lt; k < NFACES * N; k += T::TPC) {
            const int side = k / N, q = k % N, axis = side / 2;
            const int nb = neighbor(g, cell, side), face = face_of(g, cell, side);
            const double *own = wtr + ((size_t)cell * NFACES + side) * N * NVAR + q * NVAR;
            const double *oth = wtr + ((size_t)nb * NFACES + (side ^ 1)) * N * NVAR + q * NVAR;
            double z[4];
#pragma unroll
            for (int v = 0; v < NVAR; ++v) z[v] = side % 2 ? own[v] - oth[v] : oth[v] - own[v];
            const bool left = side % 2;
            const double *c = fcache + ((size_t)face * N + q) * 8;
            const double sa = speeds[2 * (face * N + q)], sb = speeds[2 * (face * N + q) + 1];
            const double pen = face_weight(g, b, face, q) * sa * sb / (sa + sb);
            double a[16];
            if (left) cached_jacobian(g.gamma, c[0], c[1], c[2], axis, a);
            else cached_jacobian(g.gamma, c[3], c[4], c[5], axis, a);
            const double blend = left ? c[6] : c[7], sp = left ? pen : -pen;
#pragma unroll
            for (int ww = 0; ww < NVAR; ++ww) {
                double s = 0;
#pragma unroll
                for (int v = 0; v < NVAR; ++v) s += a[v * 4 + ww] * z[v];
                ff[sub][k * NVAR + ww] = blend * s + sp * z[ww];
            }
        }
    __syncthreads();
    if (!active || lt >= T::P) return;
    const int ix = lt % N, iy = lt / N;
    const double mass = .25 * g.hx * g.hy * b.w[ix] * b.w[iy];
    const double sx = .5 * g.hy, sy = .5 * g.hx;
    double gx[4], gy[4];
#pragma unroll
    for (int v = 0; v < NVAR; ++v) {
        double x = 0, y = 0;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            x += b.dw[ix * N + i] * ws[sub][v * T::P + i + N * iy];
            y += b.dw[iy * N + i] * ws[sub][v * T::P + ix + N * i];
        }
        gx[v] = x;
        gy[v] = y;
    }
    const double *c = vol + ((size_t)cell * T::P + lt) * 3;
    double ax[16], ay[16];
    cached_jacobian(g.gamma, c[0], c[1], c[2], 0, ax);
    cached_jacobian(g.gamma, c[0], c[1], c[2], 1, ay);
#pragma unroll
    for (int ww = 0; ww < NVAR; ++ww) {
        double tx = 0, ty = 0;
#pragma unroll
        for (int v = 0; v < NVAR; ++v) {
            tx += ax[v * 4 + ww] * gx[v];
            ty += ay[v * 4 + ww] * gy[v];
        }
        double val = mass * ws[sub][ww * T::P + lt] * inv_step;
        if (N > 1 && volterm) val -= sx * b.w[iy] * tx + sy * b.w[ix] * ty;
        val += b.eL[ix] * ff[sub][(0 * N + iy) * NVAR + ww] + b.eR[ix] * ff[sub][(1 * N + iy) * NVAR + ww] +
               b.eL[iy] * ff[sub][(2 * N + ix) * NVAR + ww] + b.eR[iy] * ff[sub][(3 * N + ix) * NVAR + ww];
        out[base + ww * T::P + lt] = val;
    }
}

// ---- per-cell Jacobian tables used by the block assemblies ---------------------------------
// jx/jy[node*16 + v*4 + w]: physical flux Jacobians at the nodes; fj[(side*N+q)*16 + v*4 + w]:
// the face derivative per side (HLL self-coupling for DG with its lift sign, or the HDG
// derivative of face_jacobian.cpp:77-82 for condensation).
template <int N, bool HDG>
__device__ inline void cell_tables(int cell, const double *__restrict__ vol, const double *__restrict__ fcache,
                                   const double *__restrict__ speeds, const Basis1D &b, const Grid &g, double *jx,
                                   double *jy, double *fj) {
    constexpr int P = N * N;
    for (int node = threadIdx.x; node < P; node += blockDim.x) {
        const double *c = vol + ((size_t)cell * P + node) * 3;
        double a[16];
        cached_jacobian(g.gamma, c[0], c[1], c[2], 0, a);
#pragma unroll
        for (int k = 0; k < 16; ++k) jx[node * 16 + k] = a[k];
        cached_jacobian(g.gamma, c[0], c[1], c[2], 1, a);
#pragma unroll
        for (int k = 0; k < 16; ++k) jy[node * 16 + k] = a[k];
    }
    for (int k = threadIdx.x; k < NFACES * N; k += blockDim.x) {
        const int side = k / N, q = k % N, face = face_of(g, cell, side), axis = side / 2;
        const bool left = side % 2;  // this cell is the left state of faces on sides 1 and 3
        const double *c = fcache + ((size_t)face * N + q) * 8;
        const double sa = speeds[2 * (face * N + q)], sb = speeds[2 * (face * N + q) + 1];
        const double w = face_weight(g, b, face, q);
        double a[16];
        if (left) cached_jacobian(g.gamma, c[0], c[1], c[2], axis, a);
        else cached_jacobian(g.gamma, c[3], c[4], c[5], axis, a);
        if (!HDG) {  // FaceJacobian::hll (face_jacobian.cpp:69-73) times the lift sign
            const double blend = left ? c[6] : c[7], pen = w * sa * sb / (sa + sb);
            const double sign = left ? 1. : -1.;
#pragma unroll
            for (int v = 0; v < 4; ++v)
#pragma unroll
                for (int ww = 0; ww < 4; ++ww)
                    fj[k * 16 + v * 4 + ww] = sign * (a[v * 4 + ww] * blend + (v == ww ? (left ? pen : -pen) : 0.));
        } else {  // FaceJacobian::hdg: w (sign F' + tau I)
            const double sign = left ? 1. : -1., tau = left ? sa : sb;
#pragma unroll
            for (int v = 0; v < 4; ++v)
#pragma unroll
                for (int ww = 0; ww < 4; ++ww)
                    fj[k * 16 + v * 4 + ww] = (sign * a[v * 4 + ww] + (v == ww ? tau : 0.)) * w;
        }
    }
}

// Entry (row r = (v, ix, iy), col c = (w, jx, jy)) of the collocated cell block: volume part
// (volume_jacobian.cpp:72-89), the four face self-couplings (dg_operator.cpp:40-66 with
// row == col, or hybrid.cpp:31-55 for the HDG local matrix) and M/tau on the diagonal.
template <int N>
__device__ inline double cell_block_entry(int r, int c, const double *jx, const double *jy, const double *fj,
                                          const Basis1D &b, const Grid &g, double inv_step, bool volterm = true) {
    constexpr int P = N * N;
    const int v = r / P, rn = r % P, ix = rn % N, iy = rn / N;
    const int w = c / P, cn = c % P, jx_ = cn % N, jy_ = cn / N;
    double val = 0;
    const int vw = v * 4 + w;
    if (iy == jy_) {
        if (N > 1 && volterm) val -= .5 * g.hy * b.w[jy_] * jx[cn * 16 + vw] * b.dw[jx_ * N + ix];
        val += b.eL[ix] * b.eL[jx_] * fj[(0 * N + iy) * 16 + vw] + b.eR[ix] * b.eR[jx_] * fj[(1 * N + iy) * 16 + vw];
    }
    if (ix == jx_) {
        if (N > 1 && volterm) val += -.5 * g.hx * b.w[jx_] * jy[cn * 16 + vw] * b.dw[jy_ * N + iy];
        val += b.eL[iy] * b.eL[jy_] * fj[(2 * N + ix) * 16 + vw] + b.eR[iy] * b.eR[jy_] * fj[(3 * N + ix) * 16 + vw];
    }
    if (r == c) val += .25 * g.hx * g.hy * b.w[ix] * b.w[iy] * inv_step;
    return val;
}

// Copies the basis tables a kernel indexes per thread into shared memory: indexed reads of a
// kernel parameter with lane-varying indices serialise in the parameter bank, shared-memory
// reads do not.  The caller synchronises before the first use.
template <int N> __device__ inline void stage_basis(const Basis1D &b, Basis1D &sb) {
    for (int k = threadIdx.x; k < N * N; k += blockDim.x) sb.dw[k] = b.dw[k];
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
        sb.w[k] = b.w[k];
        sb.eL[k] = b.eL[k];
        sb.eR[k] = b.eR[k];
    }
}

// DG diagonal blocks written row-major into the factor pool (precision TF).  volterm = 0 leaves the
// volume term out (it is added at the over-integrated points by k_vol_block_q).
template <int N, typename TF>
__global__ void __launch_bounds__(256)
k_dg_assemble(TF *__restrict__ pool, const double *__restrict__ vol, const double *__restrict__ fcache,
              const double *__restrict__ speeds, Basis1D b, Grid g, double inv_step, int first, int count,
              int volterm = 1) {
    constexpr int P = N * N, M = NVAR * P;
    __shared__ double jx[P * 16], jy[P * 16], fj[NFACES * N * 16];
    __shared__ Basis1D sb;
    stage_basis<N>(b, sb);
    for (int blk = blockIdx.x; blk < count; blk += gridDim.x) {
        const int cell = first + blk;
        __syncthreads();
        cell_tables<N, false>(cell, vol, fcache, speeds, sb, g, jx, jy, fj);
        __syncthreads();
        TF *A = pool + (size_t)blk * M * M;
        for (int idx = threadIdx.x; idx < M * M; idx += blockDim.x)
            A[idx] = (TF)cell_block_entry<N>(idx / M, idx % M, jx, jy, fj, sb, g, inv_step, volterm != 0);
    }
}

}  // namespace dgh
