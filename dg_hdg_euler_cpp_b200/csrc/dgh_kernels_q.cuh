// Over-integrated 2D volume terms (--quad Q > k+1): the volume flux, its linearisation and the
// volume part of the cell blocks evaluated at a Q x Q Gauss rule instead of at the nodes
// (tensor_product.cpp:11-21,57-72, discretization.cpp:111-122,184-192,219-233,
// volume_jacobian.cpp:30-42,59-71,90-116).  The face terms and the mass matrix are the
// collocated ones, so the collocated kernels run with their volume part switched off and the
// kernels here add it.  One CTA per cell (grid-stride), the cell's nodal data, its values at
// the points and the two-stage tensor contractions in shared memory.
#pragma once
#include "dgh_kernels_dg.cuh"

namespace dgh {

constexpr int MAXQ2 = 16;   // volume points per direction supported on the device
constexpr int Q_THREADS = 256;

// The volume rule: V[q][i] = l_i(qx_q), wd[q][i] = qw_q l_i'(qx_q) (nodal_basis.hpp:49-56).
struct BasisQ {
    int Q;
    double V[MAXQ2 * MAXN], wd[MAXQ2 * MAXN], qw[MAXQ2];
};

// Shared scratch of one cell: nodal values, the x-interpolated half step, point values and
// the two point-flux arrays.
template <int N> struct QScratch {
    static constexpr int P = N * N;
    double nodal[NVAR * P];
    double half[NVAR * MAXQ2 * N];
    double pts[NVAR * MAXQ2 * MAXQ2];
    double fx[NVAR * MAXQ2 * MAXQ2], fy[NVAR * MAXQ2 * MAXQ2];
};

// pts[v][a + Q b] = sum_{ix, iy} V[a][ix] V[b][iy] nodal[v][ix + N iy]; ends synchronised.
template <int N>
__device__ inline void q_interpolate(const double *nodal, double *half, double *pts, const BasisQ &bq) {
    const int Q = bq.Q;
    for (int e = threadIdx.x; e < NVAR * Q * N; e += blockDim.x) {
        const int v = e / (Q * N), rem = e % (Q * N), a = rem % Q, iy = rem / Q;
        double s = 0;
#pragma unroll
        for (int ix = 0; ix < N; ++ix) s += bq.V[a * N + ix] * nodal[v * N * N + ix + N * iy];
        half[v * Q * N + a + Q * iy] = s;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < NVAR * Q * Q; e += blockDim.x) {
        const int v = e / (Q * Q), rem = e % (Q * Q), a = rem % Q, b = rem / Q;
        double s = 0;
#pragma unroll
        for (int iy = 0; iy < N; ++iy) s += half[v * Q * N + a + Q * iy] * bq.V[b * N + iy];
        pts[v * Q * Q + a + Q * b] = s;
    }
    __syncthreads();
}

// out[v][i + N j] -= (hy/2) sum_b [sum_a wd[a][i] fx(a,b)] qw[b] V[b][j]
//                  + (hx/2) sum_b [sum_a qw[a] V[a][i] fy(a,b)] wd[b][j]   (tensor_product.cpp:64-71)
// t1, t2: NVAR * N * Q scratch each (reuses half and pts of the scratch).
template <int N>
__device__ inline void q_subtract_weak(const double *fx, const double *fy, double *t1, double *t2, double *out,
                                       const BasisQ &bq, const Grid &g) {
    const int Q = bq.Q;
    for (int e = threadIdx.x; e < NVAR * N * Q; e += blockDim.x) {
        const int v = e / (N * Q), rem = e % (N * Q), i = rem % N, b = rem / N;
        double s1 = 0, s2 = 0;
        for (int a = 0; a < Q; ++a) {
            s1 += bq.wd[a * N + i] * fx[v * Q * Q + a + Q * b];
            s2 += bq.qw[a] * bq.V[a * N + i] * fy[v * Q * Q + a + Q * b];
        }
        t1[v * N * Q + i + N * b] = s1;
        t2[v * N * Q + i + N * b] = s2;
    }
    __syncthreads();
    const double sx = .5 * g.hy, sy = .5 * g.hx;
    for (int e = threadIdx.x; e < NVAR * N * N; e += blockDim.x) {
        const int v = e / (N * N), rem = e % (N * N), i = rem % N, j = rem / N;
        double s1 = 0, s2 = 0;
        for (int b = 0; b < Q; ++b) {
            s1 += t1[v * N * Q + i + N * b] * bq.qw[b] * bq.V[b * N + j];
            s2 += t2[v * N * Q + i + N * b] * bq.wd[b * N + j];
        }
        out[v * N * N + i + N * j] -= sx * s1 + sy * s2;
    }
}

template <int N> __device__ inline void q_load(const double *__restrict__ src, double *nodal) {
    for (int k = threadIdx.x; k < NVAR * N * N; k += blockDim.x) nodal[k] = src[k];
    __syncthreads();
}

// r -= the over-integrated weak volume term of F(u) (discretization.cpp:116-120).
template <int N>
__global__ void __launch_bounds__(Q_THREADS)
k_vol_residual_q(const double *__restrict__ u, double *__restrict__ r, const BasisQ *__restrict__ bqp, Grid g) {
    __shared__ QScratch<N> sc;
    __shared__ BasisQ bq;
    for (int k = threadIdx.x; k < (int)(sizeof(BasisQ) / sizeof(double)); k += blockDim.x)
        reinterpret_cast<double *>(&bq)[k] = reinterpret_cast<const double *>(bqp)[k];
    for (int cell = blockIdx.x; cell < g.cells; cell += gridDim.x) {
        __syncthreads();
        q_load<N>(u + (size_t)cell * NVAR * N * N, sc.nodal);
        q_interpolate<N>(sc.nodal, sc.half, sc.pts, bq);
        const int QQ = bq.Q * bq.Q;
        for (int q = threadIdx.x; q < QQ; q += blockDim.x) {
            const double s[4] = {sc.pts[q], sc.pts[QQ + q], sc.pts[2 * QQ + q], sc.pts[3 * QQ + q]};
            double a[4], c[4];
            flux(g.gamma, s, 0, a);
            flux(g.gamma, s, 1, c);
#pragma unroll
            for (int v = 0; v < NVAR; ++v) {
                sc.fx[v * QQ + q] = a[v];
                sc.fy[v * QQ + q] = c[v];
            }
        }
        __syncthreads();
        q_subtract_weak<N>(sc.fx, sc.fy, sc.half, sc.pts, r + (size_t)cell * NVAR * N * N, bq, g);
    }
}

// volq[(cell Q^2 + q) * 3] = (u, v, H) at the volume points (volume_jacobian.cpp:30-42).
template <int N>
__global__ void __launch_bounds__(Q_THREADS)
k_volume_cache_q(const double *__restrict__ u, double *__restrict__ volq, const BasisQ *__restrict__ bqp, Grid g) {
    __shared__ QScratch<N> sc;
    __shared__ BasisQ bq;
    for (int k = threadIdx.x; k < (int)(sizeof(BasisQ) / sizeof(double)); k += blockDim.x)
        reinterpret_cast<double *>(&bq)[k] = reinterpret_cast<const double *>(bqp)[k];
    for (int cell = blockIdx.x; cell < g.cells; cell += gridDim.x) {
        __syncthreads();
        q_load<N>(u + (size_t)cell * NVAR * N * N, sc.nodal);
        q_interpolate<N>(sc.nodal, sc.half, sc.pts, bq);
        const int QQ = bq.Q * bq.Q;
        for (int q = threadIdx.x; q < QQ; q += blockDim.x) {
            const double s[4] = {sc.pts[q], sc.pts[QQ + q], sc.pts[2 * QQ + q], sc.pts[3 * QQ + q]};
            const Prim p = primitive(g.gamma, s);
            double *c = volq + ((size_t)cell * QQ + q) * 3;
            c[0] = p.vx;
            c[1] = p.vy;
            c[2] = p.H;
        }
    }
}

// out -= the over-integrated weak term of the linearised volume flux of d (volume_jacobian.cpp:59-71).
template <int N>
__global__ void __launch_bounds__(Q_THREADS)
k_vol_apply_q(const double *__restrict__ d, const double *__restrict__ volq, double *__restrict__ out,
              const BasisQ *__restrict__ bqp, Grid g) {
    __shared__ QScratch<N> sc;
    __shared__ BasisQ bq;
    for (int k = threadIdx.x; k < (int)(sizeof(BasisQ) / sizeof(double)); k += blockDim.x)
        reinterpret_cast<double *>(&bq)[k] = reinterpret_cast<const double *>(bqp)[k];
    for (int cell = blockIdx.x; cell < g.cells; cell += gridDim.x) {
        __syncthreads();
        q_load<N>(d + (size_t)cell * NVAR * N * N, sc.nodal);
        q_interpolate<N>(sc.nodal, sc.half, sc.pts, bq);
        const int QQ = bq.Q * bq.Q;
        for (int q = threadIdx.x; q < QQ; q += blockDim.x) {
            const double dd[4] = {sc.pts[q], sc.pts[QQ + q], sc.pts[2 * QQ + q], sc.pts[3 * QQ + q]};
            const double *c = volq + ((size_t)cell * QQ + q) * 3;
            double a[4], e[4];
            normal_action(g.gamma, c[0], c[1], c[2], dd, 0, a);
            normal_action(g.gamma, c[0], c[1], c[2], dd, 1, e);
#pragma unroll
            for (int v = 0; v < NVAR; ++v) {
                sc.fx[v * QQ + q] = a[v];
                sc.fy[v * QQ + q] = e[v];
            }
        }
        __syncthreads();
        q_subtract_weak<N>(sc.fx, sc.fy, sc.half, sc.pts, out + (size_t)cell * NVAR * N * N, bq, g);
    }
}

// out -= the transpose of the over-integrated volume term of k_vol_apply_q, for the adjoint
// J^T w.  With Kx(a,b; i,j) = (hy/2) wd[a][i] qw[b] V[b][j] and Ky(a,b; i,j) = (hx/2) qw[a] V[a][i]
// wd[b][j] the forward term is sum_ab Kx Ax(a,b) I(d)(a,b) + Ky Ay(a,b) I(d)(a,b), I the
// interpolation to the points; its transpose takes the point values gx = Kx^T w, gy = Ky^T w,
// applies Ax^T gx + Ay^T gy at every point (cached_jacobian from (u, v, H) at the point) and
// returns them to the nodes with I^T.
template <int N>
__global__ void __launch_bounds__(Q_THREADS)
k_vol_apply_q_t(const double *__restrict__ w, const double *__restrict__ volq, double *__restrict__ out,
                const BasisQ *__restrict__ bqp, Grid g) {
    __shared__ QScratch<N> sc;
    __shared__ BasisQ bq;
    for (int k = threadIdx.x; k < (int)(sizeof(BasisQ) / sizeof(double)); k += blockDim.x)
        reinterpret_cast<double *>(&bq)[k] = reinterpret_cast<const double *>(bqp)[k];
    const int Q = bq.Q, QQ = Q * Q;
    const double sx = .5 * g.hy, sy = .5 * g.hx;
    for (int cell = blockIdx.x; cell < g.cells; cell += gridDim.x) {
        __syncthreads();
        q_load<N>(w + (size_t)cell * NVAR * N * N, sc.nodal);
        // hx1[v][a][j] = sum_i wd[a][i] w(i, j) (in half), hy1[v][a][j] = sum_i V[a][i] w(i, j) (in pts)
        for (int e = threadIdx.x; e < NVAR * Q * N; e += blockDim.x) {
            const int v = e / (Q * N), rem = e % (Q * N), a = rem % Q, j = rem / Q;
            double s1 = 0, s2 = 0;
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const double wv = sc.nodal[v * N * N + i + N * j];
                s1 += bq.wd[a * N + i] * wv;
                s2 += bq.V[a * N + i] * wv;
            }
            sc.half[v * Q * N + a + Q * j] = s1;
            sc.pts[v * Q * N + a + Q * j] = s2;
        }
        __syncthreads();
        // gx[v][a + Q b] = sx qw[b] sum_j V[b][j] hx1, gy[v][a + Q b] = sy qw[a] sum_j wd[b][j] hy1
        for (int e = threadIdx.x; e < NVAR * QQ; e += blockDim.x) {
            const int v = e / QQ, q = e % QQ, a = q % Q, b = q / Q;
            double s1 = 0, s2 = 0;
#pragma unroll
            for (int j = 0; j < N; ++j) {
                s1 += bq.V[b * N + j] * sc.half[v * Q * N + a + Q * j];
                s2 += bq.wd[b * N + j] * sc.pts[v * Q * N + a + Q * j];
            }
            sc.fx[v * QQ + q] = sx * bq.qw[b] * s1;
            sc.fy[v * QQ + q] = sy * bq.qw[a] * s2;
        }
        __syncthreads();
        // t(a, b) = Ax^T gx + Ay^T gy at every point (in pts)
        for (int q = threadIdx.x; q < QQ; q += blockDim.x) {
            const double *c = volq + ((size_t)cell * QQ + q) * 3;
            double ax[16], ay[16];
            cached_jacobian(g.gamma, c[0], c[1], c[2], 0, ax);
            cached_jacobian(g.gamma, c[0], c[1], c[2], 1, ay);
#pragma unroll
            for (int ww = 0; ww < NVAR; ++ww) {
                double t = 0;
#pragma unroll
                for (int v = 0; v < NVAR; ++v) t += ax[v * 4 + ww] * sc.fx[v * QQ + q] + ay[v * 4 + ww] * sc.fy[v * QQ + q];
                sc.pts[ww * QQ + q] = t;
            }
        }
        __syncthreads();
        // I^T: s1[w][k][b] = sum_a V[a][k] t(a, b) (in half), out(k, l) -= sum_b V[b][l] s1
        for (int e = threadIdx.x; e < NVAR * N * Q; e += blockDim.x) {
            const int v = e / (N * Q), rem = e % (N * Q), k = rem % N, b = rem / N;
            double s = 0;
            for (int a = 0; a < Q; ++a) s += bq.V[a * N + k] * sc.pts[v * QQ + a + Q * b];
            sc.half[v * N * Q + k + N * b] = s;
        }
        __syncthreads();
        double *o = out + (size_t)cell * NVAR * N * N;
        for (int e = threadIdx.x; e < NVAR * N * N; e += blockDim.x) {
            const int v = e / (N * N), rem = e % (N * N), k = rem % N, l = rem / N;
            double s = 0;
            for (int b = 0; b < Q; ++b) s += bq.V[b * N + l] * sc.half[v * N * Q + k + N * b];
            o[e] -= s;
        }
    }
}

// A[row * ld + col] += the over-integrated volume block (volume_jacobian.cpp:90-116) for cells
// first..first+count-1 (A chunk-relative): for each flux/state pair (v, w),
//   LX_b(k, i) = -sum_a wd[a][i] X_ab(v,w) V[a][k],  LY_b(k, i) = -sum_a qw[a] V[a][i] Y_ab(v,w) V[a][k],
//   entry (v,i,j; w,k,l) += sum_b (hy/2) qw[b] V[b][j] V[b][l] LX_b(k,i) + (hx/2) wd[b][j] V[b][l] LY_b(k,i).
template <int N, typename TF>
__global__ void __launch_bounds__(Q_THREADS)
k_vol_block_q(TF *__restrict__ A, int ld, const double *__restrict__ volq, const BasisQ *__restrict__ bqp, Grid g,
              int first, int count) {
    constexpr int P = N * N;
    __shared__ BasisQ bq;
    __shared__ double xj[MAXQ2 * MAXQ2], yj[MAXQ2 * MAXQ2];
    __shared__ double lx[MAXQ2 * P], ly[MAXQ2 * P];
    for (int k = threadIdx.x; k < (int)(sizeof(BasisQ) / sizeof(double)); k += blockDim.x)
        reinterpret_cast<double *>(&bq)[k] = reinterpret_cast<const double *>(bqp)[k];
    const int Q = bqp->Q, QQ = Q * Q;
    const double sx = .5 * g.hy, sy = .5 * g.hx;
    for (int blk = blockIdx.x; blk < count; blk += gridDim.x) {
        const int cell = first + blk;
        TF *Ab = A + (size_t)blk * NVAR * P * ld;
        for (int vw = 0; vw < 16; ++vw) {
            const int v = vw / 4, w = vw % 4;
            __syncthreads();
            for (int q = threadIdx.x; q < QQ; q += blockDim.x) {
                const double *c = volq + ((size_t)cell * QQ + q) * 3;
                double a[16];
                cached_jacobian(g.gamma, c[0], c[1], c[2], 0, a);
                xj[q] = a[v * 4 + w];
                cached_jacobian(g.gamma, c[0], c[1], c[2], 1, a);
                yj[q] = a[v * 4 + w];
            }
            __syncthreads();
            for (int e = threadIdx.x; e < Q * P; e += blockDim.x) {
                const int b = e / P, rem = e % P, k = rem / N, i = rem % N;
                double s1 = 0, s2 = 0;
                for (int a = 0; a < Q; ++a) {
                    const int q = a + Q * b;
                    s1 += bq.wd[a * N + i] * xj[q] * bq.V[a * N + k];
                    s2 += bq.qw[a] * bq.V[a * N + i] * yj[q] * bq.V[a * N + k];
                }
                lx[b * P + k * N + i] = -s1;
                ly[b * P + k * N + i] = -s2;
            }
            __syncthreads();
            for (int e = threadIdx.x; e < P * P; e += blockDim.x) {
                const int rn = e / P, cn = e % P;  // row node (i, j), column node (k, l)
                const int i = rn % N, j = rn / N, k = cn % N, l = cn / N;
                double s = 0;
                for (int b = 0; b < Q; ++b) {
                    const double vl = bq.V[b * N + l];
                    s += sx * bq.qw[b] * bq.V[b * N + j] * vl * lx[b * P + k * N + i] +
                         sy * bq.wd[b * N + j] * vl * ly[b * P + k * N + i];
                }
                TF *dst = Ab + (size_t)(v * P + rn) * ld + w * P + cn;
                *dst = (TF)((double)*dst + s);
            }
        }
    }
}

// CFL rate per cell with the volume states at the points (discretization.cpp:178-195); one
// partial maximum per CTA.
template <int N>
__global__ void __launch_bounds__(Q_THREADS)
k_rate_q(const double *__restrict__ u, const double *__restrict__ speeds, const BasisQ *__restrict__ bqp, Grid g,
         double *__restrict__ partial, int *status) {
    __shared__ QScratch<N> sc;
    __shared__ BasisQ bq;
    __shared__ double ra[Q_THREADS], rb[Q_THREADS];
    for (int k = threadIdx.x; k < (int)(sizeof(BasisQ) / sizeof(double)); k += blockDim.x)
        reinterpret_cast<double *>(&bq)[k] = reinterpret_cast<const double *>(bqp)[k];
    double best = 0;
    for (int cell = blockIdx.x; cell < g.cells; cell += gridDim.x) {
        __syncthreads();
        q_load<N>(u + (size_t)cell * NVAR * N * N, sc.nodal);
        q_interpolate<N>(sc.nodal, sc.half, sc.pts, bq);
        double ax = 0, ay = 0;
        for (int k = threadIdx.x; k < NFACES * N; k += blockDim.x) {
            const int side = k / N, q = k % N, face = face_of(g, cell, side);
            const double s = fmax(speeds[2 * (face * N + q)], speeds[2 * (face * N + q) + 1]);
            if (side < 2) ax = fmax(ax, s); else ay = fmax(ay, s);
        }
        const int QQ = bq.Q * bq.Q;
        for (int q = threadIdx.x; q < QQ; q += blockDim.x) {
            const double s[4] = {sc.pts[q], sc.pts[QQ + q], sc.pts[2 * QQ + q], sc.pts[3 * QQ + q]};
            const Prim p = primitive(g.gamma, s);
            if (!(s[0] > 0 && p.p > 0)) atomicOr(status, ST_CFL_VOLUME);
            const double c = sqrt(g.gamma * p.p * p.ir);
            ax = fmax(ax, fabs(p.vx) + c);
            ay = fmax(ay, fabs(p.vy) + c);
        }
        ra[threadIdx.x] = ax;
        rb[threadIdx.x] = ay;
        __syncthreads();
        if (threadIdx.x == 0) {
            double mx = 0, my = 0;
            for (int t = 0; t < blockDim.x; ++t) {
                mx = fmax(mx, ra[t]);
                my = fmax(my, rb[t]);
            }
            best = fmax(best, mx / g.hx + my / g.hy);
        }
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = best;
}

// Clears *ok when a state at a volume point is non-finite or has density or pressure at or
// below 1e-13 (discretization.cpp:224-227).
template <int N>
__global__ void __launch_bounds__(Q_THREADS)
k_points_check_q(const double *__restrict__ u, const BasisQ *__restrict__ bqp, Grid g, int *ok) {
    __shared__ QScratch<N> sc;
    __shared__ BasisQ bq;
    for (int k = threadIdx.x; k < (int)(sizeof(BasisQ) / sizeof(double)); k += blockDim.x)
        reinterpret_cast<double *>(&bq)[k] = reinterpret_cast<const double *>(bqp)[k];
    for (int cell = blockIdx.x; cell < g.cells; cell += gridDim.x) {
        __syncthreads();
        q_load<N>(u + (size_t)cell * NVAR * N * N, sc.nodal);
        q_interpolate<N>(sc.nodal, sc.half, sc.pts, bq);
        const int QQ = bq.Q * bq.Q;
        bool good = true;
        for (int q = threadIdx.x; q < QQ; q += blockDim.x) {
            const double s[4] = {sc.pts[q], sc.pts[QQ + q], sc.pts[2 * QQ + q], sc.pts[3 * QQ + q]};
            const bool finite = isfinite(s[0]) && isfinite(s[1]) && isfinite(s[2]) && isfinite(s[3]);
            if (!finite || s[0] <= 1e-13 || !(pressure(g.gamma, s) > 1e-13)) good = false;
        }
        if (!good) atomicExch(ok, 0);
    }
}

}  // namespace dgh
