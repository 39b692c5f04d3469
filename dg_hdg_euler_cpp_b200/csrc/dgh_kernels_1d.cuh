// The 1D DG / condensed-HDG kernels (dg_hdg_1d/src): three conserved variables, two faces per
// cell, layout [cell][var][node] (dg_hdg_1d/include/euler/types.hpp:82-108), face e joining
// cells e and e+1 periodically, and a quadrature rule of Q >= n points (over-integration when
// Q > n, nodal_basis.hpp:36-56).
//
// Work decomposition.  A 1D cell holds at most 27 unknowns, so the residual, J*v and the
// linearisation run one thread per cell with the cell's states in registers; the dense blocks
// (DG cell blocks of 3n x 3n, the augmented condensation matrix [A | B | r] of 3n x (3n+7),
// and the 3 x 3 face blocks) are factored one warp per block with lane r owning row r, and the
// block solves likewise run one warp per block.
#pragma once
#include "dgh_kernels_init.cuh"

namespace dgh {

constexpr int NV1 = 3;      // density, momentum, energy
constexpr int MAXQ1 = 20;   // quadrature points accepted on the device
constexpr int T1 = 2 * NV1; // local trace unknowns of a cell (two faces)

// Reference element with its quadrature rule, passed by value (3.1 KB).
struct Basis1Q {
    int n, Q;
    bool colloc;               // Q == n: values is the identity (nodal_basis.hpp:52-53)
    double w[MAXN], eL[MAXN], eR[MAXN];
    double values[MAXQ1 * MAXN];  // [q][i] Lagrange values at the quadrature points
    double wd[MAXQ1 * MAXN];      // [q][i] qw_q * l_i'(qx_q)
};
struct Grid1 {
    int cells;
    double h, gamma;
};

__device__ inline double pres1(double g, const double *u) { return (g - 1) * (u[2] - .5 * u[1] * u[1] / u[0]); }
// physics.cpp:7-14
__device__ inline void flux1(double g, const double *u, double *f) {
    const double v = u[1] / u[0], p = pres1(g, u);
    f[0] = u[1];
    f[1] = u[1] * v + p;
    f[2] = (u[2] + p) * v;
}
// physics.cpp:15-21, row-major (v, w)
__device__ inline void jac1(double g, const double *u, double *J) {
    const double v = u[1] / u[0], H = (u[2] + pres1(g, u)) / u[0];
    J[0] = 0; J[1] = 1; J[2] = 0;
    J[3] = .5 * (g - 3) * v * v; J[4] = (3 - g) * v; J[5] = g - 1;
    J[6] = v * (.5 * (g - 1) * v * v - H); J[7] = H - (g - 1) * v * v; J[8] = g * v;
}
__device__ inline bool phys1(double g, const double *z, double floor) { return z[0] > floor && pres1(g, z) > floor; }
// max as std::max(a, b) = (a < b) ? b : a, which keeps a when b is NaN
__device__ inline double smax(double a, double b) { return a < b ? b : a; }

template <int N> __device__ inline void load_cell1(const double *__restrict__ u, int cell, double s[NV1][N]) {
    const double *c = u + (size_t)cell * NV1 * N;
#pragma unroll
    for (int v = 0; v < NV1; ++v)
#pragma unroll
        for (int i = 0; i < N; ++i) s[v][i] = c[v * N + i];
}
template <int N> __device__ inline void sample1(const double s[NV1][N], const double *shape, double *out) {
#pragma unroll
    for (int v = 0; v < NV1; ++v) {
        double a = 0;
#pragma unroll
        for (int i = 0; i < N; ++i) a += shape[i] * s[v][i];
        out[v] = a;
    }
}
template <int N> __device__ inline void qstate1(const Basis1Q &b, const double s[NV1][N], int q, double *out) {
    if (b.colloc) {
#pragma unroll
        for (int v = 0; v < NV1; ++v) out[v] = s[v][q];
        return;
    }
    sample1<N>(s, b.values + q * N, out);
}

// r[v][i] -= sum_q wd(q,i) F[q][v]: the weak volume term (discretization.cpp:108-110).
template <int N> __device__ inline void weak_volume1(const Basis1Q &b, const double (*F)[NV1], double r[NV1][N]) {
#pragma unroll
    for (int v = 0; v < NV1; ++v)
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double a = 0;
            for (int q = 0; q < b.Q; ++q) a += b.wd[q * N + i] * F[q][v];
            r[v][i] -= a;
        }
}

// Face traces tr[cell][side][var] (side 0 = left, 1 = right) and, with CHECK, the admissibility
// test of discretization.cpp:128-144 (finite entries; rho, p > 1e-13 at nodes, quadrature
// points and both traces).
template <int N, bool CHECK>
__global__ void k1_traces(const double *__restrict__ u, double *__restrict__ tr, Basis1Q b, Grid1 g, int *ok) {
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= g.cells) return;
    double s[NV1][N];
    load_cell1<N>(u, cell, s);
    double l[NV1], r[NV1];
    sample1<N>(s, b.eL, l);
    sample1<N>(s, b.eR, r);
#pragma unroll
    for (int v = 0; v < NV1; ++v) {
        tr[(size_t)cell * T1 + v] = l[v];
        tr[(size_t)cell * T1 + NV1 + v] = r[v];
    }
    if (CHECK) {
        bool good = true;
#pragma unroll
        for (int v = 0; v < NV1; ++v)
#pragma unroll
            for (int i = 0; i < N; ++i) good = good && isfinite(s[v][i]);
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const double z[NV1] = {s[0][i], s[1][i], s[2][i]};
            good = good && phys1(g.gamma, z, 1e-13);
        }
        for (int q = 0; q < b.Q; ++q) {
            double z[NV1];
            qstate1<N>(b, s, q, z);
            good = good && phys1(g.gamma, z, 1e-13);
        }
        good = good && phys1(g.gamma, l, 1e-13) && phys1(g.gamma, r, 1e-13);
        if (!good) *ok = 0;
    }
}

// Frozen Einfeldt speeds per face (physics.cpp:25-38): speeds[2e], speeds[2e+1] = a, b.
__global__ void k1_speeds(const double *__restrict__ tr, double *__restrict__ speeds, Grid1 g, double safety,
                          int *status) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= g.cells) return;
    const int next = e + 1 == g.cells ? 0 : e + 1;
    const double *l = tr + (size_t)e * T1 + NV1, *r = tr + (size_t)next * T1;
    const double gm = g.gamma, pl = pres1(gm, l), pr = pres1(gm, r);
    if (!(l[0] > 0 && r[0] > 0 && pl > 0 && pr > 0)) {
        atomicOr(status, ST_FROZEN_FACE);
        speeds[2 * e] = speeds[2 * e + 1] = 0;
        return;
    }
    const double sl = sqrt(l[0]), sr = sqrt(r[0]);
    const double ul = l[1] / l[0], ur = r[1] / r[0];
    const double cl = sqrt(gm * pl / l[0]), cr = sqrt(gm * pr / r[0]);
    const double v = (sl * ul + sr * ur) / (sl + sr);
    const double H = (sl * (l[2] + pl) / l[0] + sr * (r[2] + pr) / r[0]) / (sl + sr);
    const double c = sqrt((gm - 1) * (H - .5 * v * v));
    speeds[2 * e] = safety * smax(smax(0.0, -ul + cl), -v + c);
    speeds[2 * e + 1] = safety * smax(smax(0.0, ur + cr), v + c);
}

// CFL rate per cell (discretization.cpp:81-89): max of the two faces' speeds and the spectral
// radius at the quadrature points, over h; one maximum per thread block into partial[].
template <int N>
__global__ void __launch_bounds__(256)
k1_rate(const double *__restrict__ u, const double *__restrict__ speeds, double *__restrict__ partial, Basis1Q b,
        Grid1 g) {
    __shared__ double red[256];
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    double alpha = 0;
    if (cell < g.cells) {
        const int prev = cell == 0 ? g.cells - 1 : cell - 1;
        alpha = smax(smax(smax(speeds[2 * prev], speeds[2 * prev + 1]), speeds[2 * cell]), speeds[2 * cell + 1]);
        double s[NV1][N];
        load_cell1<N>(u, cell, s);
        for (int q = 0; q < b.Q; ++q) {
            double z[NV1];
            qstate1<N>(b, s, q, z);
            alpha = smax(alpha, fabs(z[1] / z[0]) + sqrt(g.gamma * pres1(g.gamma, z) / z[0]));
        }
        alpha = alpha / g.h;
    }
    red[threadIdx.x] = alpha;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] = smax(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// HLL numerical flux of face e (discretization.cpp:119-120).
__device__ inline void hll1(double gm, const double *l, const double *r, double a, double bb, double *f) {
    double fl[NV1], fr[NV1];
    flux1(gm, l, fl);
    flux1(gm, r, fr);
#pragma unroll
    for (int v = 0; v < NV1; ++v) f[v] = (bb * fl[v] + a * fr[v] + a * bb * (l[v] - r[v])) / (a + bb);
}

// DG residual (discretization.cpp:102-127): M (u - old) / tau, minus the weak volume flux, plus
// the two HLL face fluxes lifted with the boundary values.  The faces are accumulated in the
// reference's face-loop order for each cell.
template <int N>
__global__ void __launch_bounds__(128)
k1_residual(const double *__restrict__ u, const double *__restrict__ old, const double *__restrict__ tr,
            const double *__restrict__ speeds, double *__restrict__ res, Basis1Q b, Grid1 g, double inv_step) {
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= g.cells) return;
    double s[NV1][N], r[NV1][N];
    load_cell1<N>(u, cell, s);
    const double *o = old + (size_t)cell * NV1 * N;
#pragma unroll
    for (int v = 0; v < NV1; ++v)
#pragma unroll
        for (int i = 0; i < N; ++i) r[v][i] = .5 * g.h * b.w[i] * (s[v][i] - o[v * N + i]) * inv_step;
    if (N > 1) {
        double F[MAXQ1][NV1];
        for (int q = 0; q < b.Q; ++q) {
            double z[NV1];
            qstate1<N>(b, s, q, z);
            flux1(g.gamma, z, F[q]);
        }
        weak_volume1<N>(b, F, r);
    }
    const int prev = cell == 0 ? g.cells - 1 : cell - 1, next = cell + 1 == g.cells ? 0 : cell + 1;
    double fp[NV1], fn[NV1];
    hll1(g.gamma, tr + (size_t)prev * T1 + NV1, tr + (size_t)cell * T1, speeds[2 * prev], speeds[2 * prev + 1], fp);
    hll1(g.gamma, tr + (size_t)cell * T1 + NV1, tr + (size_t)next * T1, speeds[2 * cell], speeds[2 * cell + 1], fn);
    double *out = res + (size_t)cell * NV1 * N;
#pragma unroll
    for (int v = 0; v < NV1; ++v)
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double x = r[v][i];
            if (cell == 0) {
                x += b.eR[i] * fn[v];
                x -= b.eL[i] * fp[v];
            } else {
                x -= b.eL[i] * fp[v];
                x += b.eR[i] * fn[v];
            }
            out[v * N + i] = x;
        }
}

// Trace lambda_e = (a l + b r + F(l) - F(r)) / (a + b) (discretization.cpp:93-101).
__global__ void k1_trace_lambda(const double *__restrict__ tr, const double *__restrict__ speeds,
                                double *__restrict__ lam, Grid1 g) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= g.cells) return;
    const int next = e + 1 == g.cells ? 0 : e + 1;
    const double *l = tr + (size_t)e * T1 + NV1, *r = tr + (size_t)next * T1;
    const double a = speeds[2 * e], bb = speeds[2 * e + 1];
    double fl[NV1], fr[NV1];
    flux1(g.gamma, l, fl);
    flux1(g.gamma, r, fr);
#pragma unroll
    for (int v = 0; v < NV1; ++v) lam[(size_t)e * NV1 + v] = (a * l[v] + bb * r[v] + fl[v] - fr[v]) / (a + bb);
}

// Linearisation (volume_jacobian.cpp:17-37, dg_operator.cpp:7-23): flux Jacobians at every
// quadrature point jq[cell][q][9], and per face the two blended face Jacobians
// fj[face][0..8] = b/(a+b) (J(l) + a I), fj[face][9..17] = a/(a+b) (J(r) - b I).
template <int N>
__global__ void __launch_bounds__(128)
k1_linearise(const double *__restrict__ u, const double *__restrict__ tr, const double *__restrict__ speeds,
             double *__restrict__ jq, double *__restrict__ fj, Basis1Q b, Grid1 g) {
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= g.cells) return;
    if (N > 1) {
        double s[NV1][N];
        load_cell1<N>(u, cell, s);
        for (int q = 0; q < b.Q; ++q) {
            double z[NV1];
            qstate1<N>(b, s, q, z);
            jac1(g.gamma, z, jq + ((size_t)cell * b.Q + q) * 9);
        }
    }
    const int next = cell + 1 == g.cells ? 0 : cell + 1;
    const double a = speeds[2 * cell], bb = speeds[2 * cell + 1];
    double jl[9], jr[9];
    jac1(g.gamma, tr + (size_t)cell * T1 + NV1, jl);
    jac1(g.gamma, tr + (size_t)next * T1, jr);
    double *f = fj + (size_t)cell * 18;
#pragma unroll
    for (int v = 0; v < NV1; ++v)
#pragma unroll
        for (int w = 0; w < NV1; ++w) {
            f[v * 3 + w] = bb / (a + bb) * (jl[v * 3 + w] + (v == w ? a : 0.));
            f[9 + v * 3 + w] = a / (a + bb) * (jr[v * 3 + w] - (v == w ? bb : 0.));
        }
}

// Matrix-free J*d (volume_jacobian.cpp:78-104, dg_operator.cpp:24-49).
template <int N>
__global__ void __launch_bounds__(128)
k1_dg_apply(const double *__restrict__ d, const double *__restrict__ jq, const double *__restrict__ fj,
            double *__restrict__ out, Basis1Q b, Grid1 g, double inv_step) {
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= g.cells) return;
    double s[NV1][N], r[NV1][N];
    load_cell1<N>(d, cell, s);
#pragma unroll
    for (int v = 0; v < NV1; ++v)
#pragma unroll
        for (int i = 0; i < N; ++i) r[v][i] = .5 * g.h * b.w[i] * s[v][i] * inv_step;
    if (N > 1) {
        double F[MAXQ1][NV1];
        for (int q = 0; q < b.Q; ++q) {
            double z[NV1];
            qstate1<N>(b, s, q, z);
            const double *J = jq + ((size_t)cell * b.Q + q) * 9;
#pragma unroll
            for (int v = 0; v < NV1; ++v) F[q][v] = J[v * 3] * z[0] + J[v * 3 + 1] * z[1] + J[v * 3 + 2] * z[2];
        }
        weak_volume1<N>(b, F, r);
    }
    const int prev = cell == 0 ? g.cells - 1 : cell - 1, next = cell + 1 == g.cells ? 0 : cell + 1;
    double sp[NV1][N], sn[NV1][N];
    load_cell1<N>(d, prev, sp);
    load_cell1<N>(d, next, sn);
    double lp[NV1], lc[NV1], rc[NV1], rn[NV1];
    sample1<N>(sp, b.eR, lp);
    sample1<N>(s, b.eL, lc);
    sample1<N>(s, b.eR, rc);
    sample1<N>(sn, b.eL, rn);
    double fp[NV1], fn[NV1];
    const double *Fp = fj + (size_t)prev * 18, *Fc = fj + (size_t)cell * 18;
#pragma unroll
    for (int v = 0; v < NV1; ++v) {
        double a = 0, c = 0;
#pragma unroll
        for (int w = 0; w < NV1; ++w) {
            a += Fp[v * 3 + w] * lp[w] + Fp[9 + v * 3 + w] * lc[w];
            c += Fc[v * 3 + w] * rc[w] + Fc[9 + v * 3 + w] * rn[w];
        }
        fp[v] = a;
        fn[v] = c;
    }
    double *o = out + (size_t)cell * NV1 * N;
#pragma unroll
    for (int v = 0; v < NV1; ++v)
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double x = r[v][i];
            if (cell == 0) {
                x += b.eR[i] * fn[v];
                x -= b.eL[i] * fp[v];
            } else {
                x -= b.eL[i] * fp[v];
                x += b.eR[i] * fn[v];
            }
            o[v * N + i] = x;
        }
}

// Volume block entry A_(v,i),(w,j) = -sum_q wd(q,i) J_q(v,w) values(q,j)
// (volume_jacobian.cpp:105-131), without the mass term.
template <int N>
__device__ inline double vol_entry1(const Basis1Q &b, const double *__restrict__ jq, int cell, int v, int i, int w,
                                    int j) {
    if (N == 1) return 0.;
    if (b.colloc) return -(jq[((size_t)cell * b.Q + j) * 9 + v * 3 + w] * b.wd[j * N + i]);
    double s = 0;
    for (int q = 0; q < b.Q; ++q) s += b.wd[q * N + i] * (jq[((size_t)cell * b.Q + q) * 9 + v * 3 + w] * b.values[q * N + j]);
    return -s;
}

// DG diagonal blocks, row-major m x m (dg_operator.cpp:50-78): volume block, the mass diagonal,
// then the left face (-eL eL^T FR_{e-1}) and the right face (+eR eR^T FL_e).
template <int N, typename TF>
__global__ void k1_dg_assemble(TF *__restrict__ pool, const double *__restrict__ jq, const double *__restrict__ fj,
                               Basis1Q b, Grid1 g, double inv_step, int first, int count) {
    constexpr int M = NV1 * N;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)count * M * M) return;
    const int cell = first + (int)(idx / (M * M)), e = (int)(idx % (M * M)), row = e / M, col = e % M;
    const int v = row / N, i = row % N, w = col / N, j = col % N;
    const int prev = cell == 0 ? g.cells - 1 : cell - 1;
    double val = vol_entry1<N>(b, jq, cell, v, i, w, j);
    if (row == col) val += .5 * g.h * b.w[i] * inv_step;
    val += -1.0 * b.eL[j] * fj[(size_t)prev * 18 + 9 + v * 3 + w] * b.eL[i];
    val += 1.0 * b.eR[j] * fj[(size_t)cell * 18 + v * 3 + w] * b.eR[i];
    pool[(size_t)(cell - first) * M * M + e] = (TF)val;
}

// Augmented condensation rows [A | B | r], row-major with ld = m + 7 (hybrid.cpp:44-76): A is
// the volume block plus sum_side shape shape^T (sign J(u_side) + stab I), B the -shape stab
// columns of the two faces, r the cell's residual.  stab = b on the left face, a on the right.
template <int N>
__global__ void k1_hdg_assemble(double *__restrict__ aug, const double *__restrict__ jq,
                                const double *__restrict__ tr, const double *__restrict__ speeds,
                                const double *__restrict__ rvol, Basis1Q b, Grid1 g, double inv_step, int first,
                                int count) {
    constexpr int M = NV1 * N, LD = M + T1 + 1;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)count * M * LD) return;
    const int cell = first + (int)(idx / (M * LD)), e = (int)(idx % (M * LD)), row = e / LD, col = e % LD;
    const int v = row / N, i = row % N;
    const int prev = cell == 0 ? g.cells - 1 : cell - 1;
    double val;
    if (col < M) {
        const int w = col / N, j = col % N;
        val = vol_entry1<N>(b, jq, cell, v, i, w, j);
        if (row == col) val += .5 * g.h * b.w[i] * inv_step;
        for (int side = 0; side < 2; ++side) {
            const double *shape = side == 0 ? b.eL : b.eR;
            const double stab = side == 0 ? speeds[2 * prev + 1] : speeds[2 * cell];
            double J[9];
            jac1(g.gamma, tr + (size_t)cell * T1 + side * NV1, J);
            const double deriv = (side == 0 ? -1.0 : 1.0) * J[v * 3 + w] + (v == w ? stab : 0.);
            val += shape[i] * shape[j] * deriv;
        }
    } else if (col < M + T1) {
        const int side = (col - M) / NV1, vv = (col - M) % NV1;
        const double *shape = side == 0 ? b.eL : b.eR;
        const double stab = side == 0 ? speeds[2 * prev + 1] : speeds[2 * cell];
        val = vv == v ? -shape[i] * stab : 0.;
    } else {
        val = rvol[(size_t)cell * M + row];
    }
    aug[idx] = val;  // chunk-relative: block (cell - first)
}

// Row-partial-pivoted LU of row-major m x ld blocks (m <= 32), one warp per block, lane r
// owning row r; the first largest |a| wins ties (Eigen's PartialPivLU and LAPACK getrf pick the
// same).  The row operations act on all ld columns, so augmented columns m..ld-1 end as
// L^{-1} P [B r]; with backsolve they are then overwritten with U^{-1} of that, i.e. A^{-1}[B r].
// perm[r] = original row of pivoted row r.  Flags: a non-finite input entry sets input_bit
// (dense_lu.hpp:12), a non-finite factor or |u_jj| <= DBL_MIN sets singular_bit (:13-15).
template <typename T>
__global__ void __launch_bounds__(128)
k1_small_lu(T *__restrict__ pool, size_t stride, int m, int ld, int count, int *__restrict__ perm, int *status,
            int input_bit, int singular_bit, int backsolve) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x / 32);
    for (int blk = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); blk < count; blk += warps) {
        T *A = pool + (size_t)blk * stride;
        bool bad_in = false;
        for (int k = lane; k < m * ld; k += 32) bad_in = bad_in || !isfinite((double)A[k]);
        if (__any_sync(0xffffffffu, bad_in)) {
            if (lane < m) perm[(size_t)blk * m + lane] = lane;  // keep every later gather in bounds
            if (lane == 0) atomicOr(status, input_bit);
            continue;
        }
        int orig = lane;
        for (int j = 0; j < m; ++j) {
            T best = T(-1);
            int bi = 0x7fffffff;
            if (lane >= j && lane < m) {
                const T a = A[(size_t)lane * ld + j];
                if (a == a) {  // a NaN never becomes the pivot
                    best = a < T(0) ? -a : a;
                    bi = lane;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const T ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
            }
            const int p = __shfl_sync(0xffffffffu, bi == 0x7fffffff ? j : bi, 0);
            if (p != j) {
                for (int c = lane; c < ld; c += 32) {
                    const T t = A[(size_t)j * ld + c];
                    A[(size_t)j * ld + c] = A[(size_t)p * ld + c];
                    A[(size_t)p * ld + c] = t;
                }
                const int oj = __shfl_sync(0xffffffffu, orig, j), op = __shfl_sync(0xffffffffu, orig, p);
                if (lane == j) orig = op;
                if (lane == p) orig = oj;
            }
            __syncwarp();
            const T pivot = A[(size_t)j * ld + j];
            if (lane > j && lane < m) {
                T *Ar = A + (size_t)lane * ld;
                const T l = pivot != T(0) ? Ar[j] / pivot : Ar[j];
                Ar[j] = l;
                const T *Aj = A + (size_t)j * ld;
                for (int c = j + 1; c < ld; ++c) Ar[c] -= l * Aj[c];
            }
            __syncwarp();
        }
        bool bad = false;
        for (int k = lane; k < m * m; k += 32) bad = bad || !isfinite((double)A[(size_t)(k / m) * ld + k % m]);
        if (lane < m) {
            const double d = (double)A[(size_t)lane * ld + lane];
            bad = bad || !(fabs(d) > 2.2250738585072014e-308);
            perm[(size_t)blk * m + lane] = orig;
        }
        if (__any_sync(0xffffffffu, bad)) {
            if (lane == 0) atomicOr(status, singular_bit);
            continue;
        }
        if (backsolve)
            for (int j = m - 1; j >= 0; --j) {
                const T ujj = A[(size_t)j * ld + j];
                for (int c = m + lane; c < ld; c += 32) A[(size_t)j * ld + c] /= ujj;
                __syncwarp();
                if (lane < j) {
                    T *Ar = A + (size_t)lane * ld;
                    const T l = Ar[j];
                    const T *Aj = A + (size_t)j * ld;
                    for (int c = m; c < ld; ++c) Ar[c] -= l * Aj[c];
                }
                __syncwarp();
            }
    }
}

// z = A^{-1} x per block with the factors of k1_small_lu (ld = m): y = P x, unit-lower then
// upper triangular solves with one warp per block and lane r owning row r (m <= 32).  T is the
// factor and arithmetic precision; x and z are FP64.  With transpose, z = A^{-T} x =
// P^T L^{-T} U^{-T} x instead.
template <typename T>
__global__ void __launch_bounds__(128)
k1_small_solve(const T *__restrict__ pool, const int *__restrict__ perm, int m, int count,
               const double *__restrict__ x, double *__restrict__ z, int transpose) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x / 32);
    for (int blk = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); blk < count; blk += warps) {
        const T *A = pool + (size_t)blk * m * m;
        const int *pm = perm + (size_t)blk * m;
        const bool act = lane < m;
        if (!transpose) {
            T y = act ? (T)x[(size_t)blk * m + pm[lane]] : T(0);
            for (int j = 0; j < m; ++j) {
                const T yj = __shfl_sync(0xffffffffu, y, j);
                if (act && lane > j) y -= A[(size_t)lane * m + j] * yj;
            }
            for (int j = m - 1; j >= 0; --j) {
                if (lane == j) y = y / A[(size_t)j * m + j];
                const T yj = __shfl_sync(0xffffffffu, y, j);
                if (act && lane < j) y -= A[(size_t)lane * m + j] * yj;
            }
            if (act) z[(size_t)blk * m + lane] = (double)y;
        } else {
            // U^T w = x (lower with U's diagonal), L^T v = w (unit upper), z[perm[r]] = v[r]
            T y = act ? (T)x[(size_t)blk * m + lane] : T(0);
            for (int j = 0; j < m; ++j) {
                if (lane == j) y = y / A[(size_t)j * m + j];
                const T yj = __shfl_sync(0xffffffffu, y, j);
                if (act && lane > j) y -= A[(size_t)j * m + lane] * yj;
            }
            for (int j = m - 1; j >= 0; --j) {
                const T yj = __shfl_sync(0xffffffffu, y, j);
                if (act && lane < j) y -= A[(size_t)j * m + lane] * yj;
            }
            if (act) z[(size_t)blk * m + pm[lane]] = (double)y;
        }
    }
}

// From the solved augmented rows: S = -C X (6 x 6, row-major), cy = C y, the persistent X
// (m x 6 row-major) and y (hybrid.cpp:72-83).  C(side*3 + w, (v,i)) = shape_side[i] deriv_side(w,v).
template <int N>
__global__ void k1_hdg_schur(const double *__restrict__ aug, const double *__restrict__ tr,
                             const double *__restrict__ speeds, double *__restrict__ S, double *__restrict__ X,
                             double *__restrict__ y, double *__restrict__ cy, Basis1Q b, Grid1 g, int first,
                             int count) {
    constexpr int M = NV1 * N, LD = M + T1 + 1;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= count * T1 * (T1 + 1)) return;
    const int blk = idx / (T1 * (T1 + 1)), cell = first + blk, e = idx % (T1 * (T1 + 1)), a = e / (T1 + 1),
              col = e % (T1 + 1);
    const int side = a / NV1, w = a % NV1;
    const int prev = cell == 0 ? g.cells - 1 : cell - 1;
    const double *shape = side == 0 ? b.eL : b.eR;
    const double stab = side == 0 ? speeds[2 * prev + 1] : speeds[2 * cell];
    double J[9];
    jac1(g.gamma, tr + (size_t)cell * T1 + side * NV1, J);
    const double *A = aug + (size_t)blk * M * LD;
    double s = 0;
    for (int v = 0; v < NV1; ++v) {
        const double deriv = (side == 0 ? -1.0 : 1.0) * J[w * 3 + v] + (v == w ? stab : 0.);
        for (int i = 0; i < N; ++i) s += shape[i] * deriv * A[(size_t)(v * N + i) * LD + M + col];
    }
    if (col < T1) S[(size_t)cell * T1 * T1 + a * T1 + col] = -s;
    else cy[(size_t)cell * T1 + a] = s;
    if (a == 0)
        for (int r = 0; r < M; ++r) {
            const double val = A[(size_t)r * LD + M + col];
            if (col < T1) X[((size_t)cell * M + r) * T1 + col] = val;
            else y[(size_t)cell * M + r] = val;
        }
}

// rhs_e = (C y)_{cell e, right} + (C y)_{cell e+1, left} (hybrid.cpp:46,79-82).
__global__ void k1_hdg_rhs(const double *__restrict__ cy, double *__restrict__ rhs, Grid1 g) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= g.cells * NV1) return;
    const int e = idx / NV1, v = idx % NV1, next = e + 1 == g.cells ? 0 : e + 1;
    const double right = cy[(size_t)e * T1 + NV1 + v], left = cy[(size_t)next * T1 + v];
    rhs[idx] = e + 1 == g.cells ? (-0. + left) + right : (-0. + right) + left;
}

// Schur action y_e = -(a+b) x_e + S_e[right rows] g_e + S_{e+1}[left rows] g_{e+1}
// (hybrid.cpp:85-103), g_c = (x_{c-1}, x_c) the cell's two face traces; the two cell
// contributions are added in the reference's cell-loop order.
__global__ void k1_hdg_apply(const double *__restrict__ S, const double *__restrict__ speeds,
                             const double *__restrict__ x, double *__restrict__ out, Grid1 g) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= g.cells * NV1) return;
    const int e = idx / NV1, v = idx % NV1;
    const int prev = e == 0 ? g.cells - 1 : e - 1, next = e + 1 == g.cells ? 0 : e + 1;
    const double val = -(speeds[2 * e] + speeds[2 * e + 1]) * x[idx];
    // cell e: its right face is e (rows 3..5); cell e+1: its left face is e (rows 0..2)
    const double *Se = S + (size_t)e * T1 * T1 + (NV1 + v) * T1, *Sn = S + (size_t)next * T1 * T1 + v * T1;
    const double ge[T1] = {x[(size_t)prev * NV1], x[(size_t)prev * NV1 + 1], x[(size_t)prev * NV1 + 2],
                           x[(size_t)e * NV1], x[(size_t)e * NV1 + 1], x[(size_t)e * NV1 + 2]};
    const double gn[T1] = {x[(size_t)e * NV1], x[(size_t)e * NV1 + 1], x[(size_t)e * NV1 + 2],
                           x[(size_t)next * NV1], x[(size_t)next * NV1 + 1], x[(size_t)next * NV1 + 2]};
    double a = 0, c = 0;
#pragma unroll
    for (int k = 0; k < T1; ++k) {
        a += Se[k] * ge[k];
        c += Sn[k] * gn[k];
    }
    out[idx] = e + 1 == g.cells ? (val + c) + a : (val + a) + c;
}

// Face blocks D + S_e[right, right] + S_{e+1}[left, left], row-major 3 x 3 (hybrid.cpp:104-117).
template <typename TF>
__global__ void k1_face_blocks(const double *__restrict__ S, const double *__restrict__ speeds,
                               TF *__restrict__ pool, Grid1 g) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= g.cells * 9) return;
    const int e = idx / 9, i = (idx % 9) / 3, j = idx % 3, next = e + 1 == g.cells ? 0 : e + 1;
    double val = i == j ? -(speeds[2 * e] + speeds[2 * e + 1]) : 0.;
    val += S[(size_t)e * T1 * T1 + (NV1 + i) * T1 + NV1 + j];
    val += S[(size_t)next * T1 * T1 + i * T1 + j];
    pool[idx] = (TF)val;
}

// Recovery du = -y - X g (hybrid.cpp:131-138).
template <int N>
__global__ void k1_hdg_recover(const double *__restrict__ X, const double *__restrict__ y,
                               const double *__restrict__ dl, double *__restrict__ du, Grid1 g) {
    constexpr int M = NV1 * N;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)g.cells * M) return;
    const int cell = (int)(idx / M), r = (int)(idx % M), prev = cell == 0 ? g.cells - 1 : cell - 1;
    const double *Xr = X + (size_t)idx * T1;
    double s = 0;
#pragma unroll
    for (int k = 0; k < NV1; ++k) s += Xr[k] * dl[(size_t)prev * NV1 + k];
#pragma unroll
    for (int k = 0; k < NV1; ++k) s += Xr[NV1 + k] * dl[(size_t)cell * NV1 + k];
    du[idx] = -y[idx] - s;
}

// The DG residual implied by a Schur error e (hybrid.cpp:118-130): per cell -B (e / -(a+b)),
// B(row(v,i), side*3+v) = -shape_side[i] stab_side.
template <int N>
__global__ void k1_hdg_recovered_residual(const double *__restrict__ e, const double *__restrict__ speeds,
                                          double *__restrict__ out, Basis1Q b, Grid1 g) {
    constexpr int M = NV1 * N;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)g.cells * M) return;
    const int cell = (int)(idx / M), r = (int)(idx % M), v = r / N, i = r % N;
    const int prev = cell == 0 ? g.cells - 1 : cell - 1;
    const double gl = e[(size_t)prev * NV1 + v] / -(speeds[2 * prev] + speeds[2 * prev + 1]);
    const double gr = e[(size_t)cell * NV1 + v] / -(speeds[2 * cell] + speeds[2 * cell + 1]);
    const double bl = -b.eL[i] * speeds[2 * prev + 1], br = -b.eR[i] * speeds[2 * cell];
    out[idx] = -(bl * gl + br * gr);
}

// Projected initial state with the convex positivity limiter (discretization.cpp:31-74), one
// thread per cell, on the max(20, 2n+3)-point error rule.
template <int N>
__global__ void __launch_bounds__(64)
k1_initial(double *__restrict__ u, const ErrorRule *__restrict__ er, Basis1Q b, Grid1 g, Case cs, int *status) {
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= g.cells) return;
    const int Qe = er->Q;
    double nodal[NV1][N];
#pragma unroll
    for (int v = 0; v < NV1; ++v)
#pragma unroll
        for (int i = 0; i < N; ++i) nodal[v][i] = 0;
    for (int q = 0; q < Qe; ++q) {
        double s[4];
        if (!exact_state(cs, -1 + g.h * (cell + .5) + .5 * g.h * er->ex[q], 0., 0., s)) atomicOr(status, ST_SHOCK);
        const double z[NV1] = {s[0], s[1], s[3]};
#pragma unroll
        for (int v = 0; v < NV1; ++v)
#pragma unroll
            for (int i = 0; i < N; ++i) nodal[v][i] += er->proj[i * Qe + q] * z[v];
    }
    double mean[NV1];
#pragma unroll
    for (int v = 0; v < NV1; ++v) {
        double s = 0;
#pragma unroll
        for (int i = 0; i < N; ++i) s += nodal[v][i] * b.w[i];
        mean[v] = .5 * s;
    }
    if (!(mean[0] > 0 && pres1(g.gamma, mean) > 0)) atomicOr(status, ST_NONPHYS_MEAN);
    double theta = 1;
    auto visit = [&](const double *z0) {
        double d[NV1];
        for (int v = 0; v < NV1; ++v) d[v] = z0[v] - mean[v];
        auto physical = [&](double f) {
            double z[NV1];
            for (int v = 0; v < NV1; ++v) z[v] = mean[v] + f * d[v];
            return phys1(g.gamma, z, 1e-12);
        };
        if (!physical(theta)) {
            double low = 0, high = theta;
            for (int k = 0; k < 60; ++k) {
                const double mid = .5 * (low + high);
                if (physical(mid)) low = mid;
                else high = mid;
            }
            theta = .99 * low;
        }
    };
    for (int i = 0; i < N; ++i) {
        const double z[NV1] = {nodal[0][i], nodal[1][i], nodal[2][i]};
        visit(z);
    }
    for (int q = 0; q < b.Q; ++q) {
        double z[NV1];
        sample1<N>(nodal, b.values + q * N, z);
        visit(z);
    }
    for (int q = 0; q < Qe; ++q) {
        double z[NV1];
        sample1<N>(nodal, er->ev + q * N, z);
        visit(z);
    }
    double z[NV1];
    sample1<N>(nodal, b.eL, z);
    visit(z);
    sample1<N>(nodal, b.eR, z);
    visit(z);
    double *o = u + (size_t)cell * NV1 * N;
#pragma unroll
    for (int v = 0; v < NV1; ++v)
#pragma unroll
        for (int i = 0; i < N; ++i) o[v * N + i] = mean[v] + theta * (nodal[v][i] - mean[v]);
}

// partial[cell*4+v] = .5 h sum_q ew_q (u_h - u_exact)^2 (discretization.cpp:156-168); slot 3 is 0.
template <int N>
__global__ void k1_l2_error(const double *__restrict__ u, const ErrorRule *__restrict__ er, Grid1 g, Case cs,
                            double t, double *__restrict__ partial, int *status) {
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= g.cells) return;
    double s[NV1][N];
    load_cell1<N>(u, cell, s);
    double acc[NV1] = {0, 0, 0};
    for (int q = 0; q < er->Q; ++q) {
        double ex[4], z[NV1];
        if (!exact_state(cs, -1 + g.h * (cell + .5) + .5 * g.h * er->ex[q], 0., t, ex)) atomicOr(status, ST_SHOCK);
        sample1<N>(s, er->ev + q * N, z);
        const double e3[NV1] = {ex[0], ex[1], ex[3]};
#pragma unroll
        for (int v = 0; v < NV1; ++v) acc[v] += .5 * g.h * er->ew[q] * (z[v] - e3[v]) * (z[v] - e3[v]);
    }
#pragma unroll
    for (int v = 0; v < NV1; ++v) partial[(size_t)cell * 4 + v] = acc[v];
    partial[(size_t)cell * 4 + 3] = 0;
}

// partial[cell*4+v] = sum_i .5 h w_i u (discretization.cpp:148-155); slot 3 is 0.
template <int N>
__global__ void k1_integral(const double *__restrict__ u, Basis1Q b, Grid1 g, double *__restrict__ partial) {
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= g.cells) return;
#pragma unroll
    for (int v = 0; v < NV1; ++v) {
        double s = 0;
#pragma unroll
        for (int i = 0; i < N; ++i) s += .5 * g.h * b.w[i] * u[(size_t)cell * NV1 * N + v * N + i];
        partial[(size_t)cell * 4 + v] = s;
    }
    partial[(size_t)cell * 4 + 3] = 0;
}

// Diagonal mass .5 h w_i and its inverse; the HDG GMRES metric is the identity in 1D
// (dg_hdg_1d/src/time_integrator.cpp:27).
__global__ void k1_fill_mass(double *mass, double *inv_mass, double *trace_weights, Basis1Q b, Grid1 g, int n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < (long long)g.cells * NV1 * n) {
        const double m = .5 * g.h * b.w[i % n];
        mass[i] = m;
        inv_mass[i] = 1 / m;
    }
    if (i < (long long)g.cells * NV1) trace_weights[i] = 1.;
}

}  // namespace dgh
