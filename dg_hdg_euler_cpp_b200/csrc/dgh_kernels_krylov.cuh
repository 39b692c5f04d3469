// Device-resident Arnoldi pieces of the restarted, right-preconditioned GMRES(m) with
// classical Gram-Schmidt applied twice and a weighted inner product (gmres.cpp:17-86).
// Reductions are deterministic: a fixed grid writes per-block partial sums, and k_reduce adds
// them in a fixed tree order.  The two CGS2 passes are fused so the basis is swept three times
// per iteration instead of four: dot | axpy+dot | axpy+norm.  The sweeps read 16-byte pairs
// (the basis rows, the work vectors and the metric are 16-byte aligned device buffers); an odd
// last element is handled by thread 0 of block 0.
#pragma once
#include "dgh_common.cuh"

namespace dgh {

constexpr int KR_THREADS = 256;
constexpr int KR_MAXK = 32;

// Bodies take their block index bx and block count G explicitly, so the batched kernels of a
// lockstep batch (dgh_kernels_lockstep.cuh) run exactly the arithmetic of the single-problem
// kernels on each member's own partition.
template <int NV>
__device__ inline void block_reduce_store(double (&acc)[NV], int K, double *partial, int G, int bx) {
    __shared__ double red[KR_MAXK][KR_THREADS / 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        if (k >= K) break;
        double v = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0;
#pragma unroll
        for (int w = 0; w < KR_THREADS / 32; ++w) s += red[threadIdx.x][w];
        partial[(size_t)threadIdx.x * G + bx] = s;
    }
}

// partial[k*G + blk] = sum_i V_k[i] W[i] x[i], k < K
template <int NV>
__device__ __forceinline__ void mdot_body(int bx, int G, const double *__restrict__ V, size_t ldv, int K,
                                          const double *__restrict__ x, const double *__restrict__ W, long long n,
                                          double *__restrict__ partial) {
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0;
    const long long n2 = n >> 1;
    const double2 *x2 = reinterpret_cast<const double2 *>(x), *W2 = reinterpret_cast<const double2 *>(W);
    for (long long i = (long long)bx * KR_THREADS + threadIdx.x; i < n2; i += (long long)G * KR_THREADS) {
        const double2 xv = x2[i], wv = W2[i];
        const double wx0 = rmul(wv.x, xv.x), wx1 = rmul(wv.y, xv.y);
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            const double2 v = reinterpret_cast<const double2 *>(V + k * ldv)[i];
            acc[k] = rfma(v.x, wx0, acc[k]);
            acc[k] = rfma(v.y, wx1, acc[k]);
        }
    }
    if ((n & 1) && bx == 0 && threadIdx.x == 0) {
        const long long i = n - 1;
        const double wx = rmul(W[i], x[i]);
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[k] = rfma(V[k * ldv + i], wx, acc[k]);
    }
    block_reduce_store<NV>(acc, K, partial, G, bx);
}
template <int NV>
__global__ void __launch_bounds__(KR_THREADS)
k_mdot(const double *__restrict__ V, size_t ldv, int K, const double *__restrict__ x,
       const double *__restrict__ W, long long n, double *__restrict__ partial) {
    mdot_body<NV>(blockIdx.x, gridDim.x, V, ldv, K, x, W, n, partial);
}

// x -= sum_k V_k h_k, then partial dots of the updated x with every V_k (MODE 0) or the
// weighted squared norm of the updated x (MODE 1).
template <int NV, int MODE>
__device__ __forceinline__ void maxpy_body(int bx, int G, const double *__restrict__ V, size_t ldv, int K,
                                           const double *__restrict__ h, double *__restrict__ x,
                                           const double *__restrict__ W, long long n, double *__restrict__ partial) {
    __shared__ double hs[KR_MAXK];
    if (threadIdx.x < K) hs[threadIdx.x] = h[threadIdx.x];
    __syncthreads();
    double acc[MODE == 0 ? NV : 1];
#pragma unroll
    for (int k = 0; k < (MODE == 0 ? NV : 1); ++k) acc[k] = 0;
    auto one = [&](long long i) {
        double v[NV];
        double s = 0;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            v[k] = V[k * ldv + i];
            s = rfma(v[k], hs[k], s);
        }
        const double xn = rsub(x[i], s);
        x[i] = xn;
        const double wx = rmul(W[i], xn);
        if (MODE == 0) {
#pragma unroll
            for (int k = 0; k < NV; ++k) acc[k] = rfma(v[k], wx, acc[k]);
        } else {
            acc[0] = rfma(xn, wx, acc[0]);
        }
    };
    const long long n2 = n >> 1;
    double2 *x2 = reinterpret_cast<double2 *>(x);
    const double2 *W2 = reinterpret_cast<const double2 *>(W);
    for (long long i = (long long)bx * KR_THREADS + threadIdx.x; i < n2; i += (long long)G * KR_THREADS) {
        double2 v[NV];
        double s0 = 0, s1 = 0;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            v[k] = reinterpret_cast<const double2 *>(V + k * ldv)[i];
            s0 = rfma(v[k].x, hs[k], s0);
            s1 = rfma(v[k].y, hs[k], s1);
        }
        double2 xv = x2[i];
        xv.x = rsub(xv.x, s0);
        xv.y = rsub(xv.y, s1);
        x2[i] = xv;
        const double2 wv = W2[i];
        const double wx0 = rmul(wv.x, xv.x), wx1 = rmul(wv.y, xv.y);
        if (MODE == 0) {
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                acc[k] = rfma(v[k].x, wx0, acc[k]);
                acc[k] = rfma(v[k].y, wx1, acc[k]);
            }
        } else {
            acc[0] = rfma(xv.x, wx0, acc[0]);
            acc[0] = rfma(xv.y, wx1, acc[0]);
        }
    }
    if ((n & 1) && bx == 0 && threadIdx.x == 0) one(n - 1);
    block_reduce_store<MODE == 0 ? NV : 1>(acc, MODE == 0 ? K : 1, partial, G, bx);
}
template <int NV, int MODE>
__global__ void __launch_bounds__(KR_THREADS)
k_maxpy_reduce(const double *__restrict__ V, size_t ldv, int K, const double *__restrict__ h,
               double *__restrict__ x, const double *__restrict__ W, long long n, double *__restrict__ partial) {
    maxpy_body<NV, MODE>(blockIdx.x, gridDim.x, V, ldv, K, h, x, W, n, partial);
}

// out[k] = sum_b partial[k*G + b]  (one CTA per k, fixed order)
__device__ __forceinline__ void reduce_body(int k, const double *__restrict__ partial, int G, double *__restrict__ out) {
    __shared__ double red[KR_THREADS / 32];
    double s = 0;
    for (int b = threadIdx.x; b < G; b += KR_THREADS) s += partial[(size_t)k * G + b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < KR_THREADS / 32; ++w) t += red[w];
        out[k] = t;
    }
}
__global__ void __launch_bounds__(KR_THREADS) k_reduce(const double *__restrict__ partial, int G, double *__restrict__ out) {
    reduce_body(blockIdx.x, partial, G, out);
}

// out[i] = sum_k V_k[i] c_k
template <int NV>
__global__ void __launch_bounds__(KR_THREADS)
k_lincomb(const double *__restrict__ V, size_t ldv, int K, const double *__restrict__ c, double *__restrict__ out,
          long long n) {
    __shared__ double cs[KR_MAXK];
    if (threadIdx.x < K) cs[threadIdx.x] = c[threadIdx.x];
    __syncthreads();
    const long long n2 = n >> 1;
    for (long long i = (long long)blockIdx.x * KR_THREADS + threadIdx.x; i < n2; i += (long long)gridDim.x * KR_THREADS) {
        double s0 = 0, s1 = 0;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            const double2 v = reinterpret_cast<const double2 *>(V + k * ldv)[i];
            s0 += v.x * cs[k];
            s1 += v.y * cs[k];
        }
        reinterpret_cast<double2 *>(out)[i] = make_double2(s0, s1);
    }
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        double s = 0;
#pragma unroll
        for (int k = 0; k < NV; ++k) s += V[k * ldv + n - 1] * cs[k];
        out[n - 1] = s;
    }
}

// out = x / s  when s > 0 (s read on the device: the norm of the preceding reduction)
__device__ __forceinline__ void scale_div_body(int bx, int G, const double *__restrict__ x, const double *__restrict__ s2,
                                               int sqrt_first, double *__restrict__ out, long long n) {
    const double s = sqrt_first ? sqrt(fmax(0., *s2)) : *s2;
    if (!(s > 0)) return;
    for (long long i = (long long)bx * blockDim.x + threadIdx.x; i < n; i += (long long)G * blockDim.x)
        out[i] = x[i] / s;
}
__global__ void k_scale_div(const double *__restrict__ x, const double *__restrict__ s2, int sqrt_first,
                            double *__restrict__ out, long long n) {
    scale_div_body(blockIdx.x, gridDim.x, x, s2, sqrt_first, out, n);
}

// y = a*x + b*y  (general axpby used for x += z, r = rhs - Ax, trial = state + theta*dir)
__device__ __forceinline__ void axpby_body(int bx, int G, double a, const double *x, double b, const double *y,
                                           double *out, long long n) {
    for (long long i = (long long)bx * blockDim.x + threadIdx.x; i < n; i += (long long)G * blockDim.x)
        out[i] = rfma(a, x[i], rmul(b, y[i]));
}
__global__ void k_axpby(double a, const double *x, double b, const double *y, double *out, long long n) {
    axpby_body(blockIdx.x, gridDim.x, a, x, b, y, out, n);
}

// weighted squared norm partials: sum x^2 * W  (W = inverse mass, mass, or inverse trace mass)
__device__ __forceinline__ void wnorm2_body(int bx, int G, const double *__restrict__ x, const double *__restrict__ W,
                                            int divide, long long n, double *__restrict__ partial) {
    double acc[1] = {0};
    for (long long i = (long long)bx * KR_THREADS + threadIdx.x; i < n; i += (long long)G * KR_THREADS)
        acc[0] = divide ? radd(acc[0], rmul(x[i], x[i]) / W[i]) : rfma(rmul(x[i], x[i]), W[i], acc[0]);
    block_reduce_store<1>(acc, 1, partial, G, bx);
}
__global__ void __launch_bounds__(KR_THREADS)
k_wnorm2(const double *__restrict__ x, const double *__restrict__ W, int divide, long long n,
         double *__restrict__ partial) {
    wnorm2_body(blockIdx.x, gridDim.x, x, W, divide, n, partial);
}

// out = a * M x + b * y  (M the diagonal mass matrix)
__global__ void k_mass_axpby(double a, const double *x, const double *mass, double b, const double *y, double *out,
                             long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = a * (mass[i] * x[i]) + b * y[i];
}

// Objective sum M rho^2 over the density sheets (partials) and its gradient 2 M rho (0 elsewhere).
__global__ void __launch_bounds__(KR_THREADS)
k_rho2(const double *__restrict__ u, const double *__restrict__ mass, int plane, long long n, double *__restrict__ grad,
       double *__restrict__ partial) {
    double acc[1] = {0};
    for (long long i = (long long)blockIdx.x * KR_THREADS + threadIdx.x; i < n; i += (long long)gridDim.x * KR_THREADS) {
        const bool rho = ((i / plane) % 4) == 0;
        const double v = rho ? u[i] : 0.;
        acc[0] += mass[i] * v * v;
        if (grad) grad[i] = 2. * mass[i] * v;
    }
    block_reduce_store<1>(acc, 1, partial, gridDim.x, blockIdx.x);
}

// ---- Device-resident GMRES control (gmres.cpp:24-86): the Hessenberg column, the Givens
// rotations, the inner-loop break and the least-squares back substitution run in one-thread
// kernels, so a whole restart cycle can be replayed as one CUDA graph whose Arnoldi steps are
// conditional nodes (the break of gmres.cpp:65-67 sets the condition to zero).  The same kernels
// run when the cycle is launched step by step, so both ways give the same numbers.  Each step's
// conditional node has its own handle, set by the kernel that precedes the step.
struct GmresDev {
    double H[(KR_MAXK + 1) * KR_MAXK];  // column-major, leading dimension KR_MAXK + 1
    double cs[KR_MAXK], sn[KR_MAXK], g[KR_MAXK + 1], y[KR_MAXK];
    double rhs_norm, tol, beta, rnorm2;
    int iters, limit, count, cont, status, restart;
};

// Cycle start: beta = ||r|| (from the reduction at nrm2), g = beta e_1, and whether to iterate
// (gmres.cpp:25-27 and the loop condition of :33).
__device__ __forceinline__ int gmres_init_body(GmresDev *d, const double *nrm2) {
    const double beta = sqrt(fmax(0., *nrm2));
    d->beta = beta;
    for (int i = 0; i < (KR_MAXK + 1) * KR_MAXK; ++i) d->H[i] = 0.;
    for (int i = 0; i <= KR_MAXK; ++i) d->g[i] = 0.;
    d->g[0] = beta;
    d->count = 0;
    const int cont = !(beta <= d->tol * d->rhs_norm) && d->restart > 0 && d->iters < d->limit;
    d->cont = cont;
    return cont;
}
__global__ void k_gmres_init(GmresDev *d, const double *nrm2, cudaGraphConditionalHandle h, int use_h) {
    if (threadIdx.x != 0) return;
    const int cont = gmres_init_body(d, nrm2);
    if (use_h) cudaGraphSetConditional(h, cont);
}

// After the CGS2 sweeps of step j: column j of H from the two projections (red[0..j],
// red[KR_MAXK..]) and the norm (red[2 KR_MAXK]), the earlier rotations, the new rotation, the
// rotated right-hand side and the break test (gmres.cpp:42-67).  In a captured cycle h is the
// handle of step j+1's conditional node.
__device__ __forceinline__ int gmres_update_body(GmresDev *d, const double *red, int j) {
    constexpr int LDH = KR_MAXK + 1;
    double *H = d->H + (size_t)j * LDH;
    for (int i = 0; i <= j; ++i) H[i] = (0. + red[i]) + red[KR_MAXK + i];
    const double next = sqrt(fmax(0., red[2 * KR_MAXK]));
    H[j + 1] = next;
    for (int i = 0; i < j; ++i) {
        const double a = H[i], b = H[i + 1];
        H[i] = rfma(d->cs[i], a, rmul(d->sn[i], b));
        H[i + 1] = rfma(-d->sn[i], a, rmul(d->cs[i], b));
    }
    const double dd = hypot(H[j], H[j + 1]);
    if (!(isfinite(dd) && dd > 0)) {  // "GMRES Arnoldi breakdown", reported by the host
        d->status = 1;
        d->cont = 0;
        return 0;
    }
    d->cs[j] = H[j] / dd;
    d->sn[j] = H[j + 1] / dd;
    H[j] = dd;
    H[j + 1] = 0;
    d->g[j + 1] = -d->sn[j] * d->g[j];
    d->g[j] *= d->cs[j];
    d->iters += 1;
    d->count = j + 1;
    const int cont = !(fabs(d->g[j + 1]) <= d->tol * d->rhs_norm || next <= 2.2250738585072014e-308) &&
                     j + 1 < d->restart && d->iters < d->limit;
    d->cont = cont;
    return cont;
}
__global__ void k_gmres_update(GmresDev *d, const double *red, int j, cudaGraphConditionalHandle h, int use_h) {
    if (threadIdx.x != 0) return;
    const int cont = gmres_update_body(d, red, j);
    if (use_h) cudaGraphSetConditional(h, cont);
}

// y = H(0:count, 0:count)^{-1} g (gmres.cpp:69-74); coef = y padded with zeros.
__device__ __forceinline__ void gmres_backsolve_body(GmresDev *d, double *coef) {
    constexpr int LDH = KR_MAXK + 1;
    const int cnt = d->count;
    for (int i = cnt - 1; i >= 0; --i) {
        double value = d->g[i];
        for (int jj = i + 1; jj < cnt; ++jj) value = rfma(-d->H[(size_t)jj * LDH + i], d->y[jj], value);
        d->y[i] = value / d->H[(size_t)i * LDH + i];
    }
    for (int k = 0; k < KR_MAXK; ++k) coef[k] = k < cnt ? d->y[k] : 0.;
}
__global__ void k_gmres_backsolve(GmresDev *d, double *coef) {
    if (threadIdx.x != 0) return;
    gmres_backsolve_body(d, coef);
}

// out[i] = sum_{k < *count} V_k[i] c_k with the basis size read on the device.
__device__ __forceinline__ void lincomb_dyn_body(int bx, int G, const double *__restrict__ V, size_t ldv,
                                                 const int *countp, const double *__restrict__ c,
                                                 double *__restrict__ out, long long n) {
    __shared__ double cs[KR_MAXK];
    const int K = *countp;
    if (threadIdx.x < KR_MAXK) cs[threadIdx.x] = threadIdx.x < K ? c[threadIdx.x] : 0.;
    __syncthreads();
    const long long n2 = n >> 1;
    for (long long i = (long long)bx * KR_THREADS + threadIdx.x; i < n2; i += (long long)G * KR_THREADS) {
        double s0 = 0, s1 = 0;
        for (int k = 0; k < K; ++k) {
            const double2 v = reinterpret_cast<const double2 *>(V + k * ldv)[i];
            s0 = rfma(v.x, cs[k], s0);
            s1 = rfma(v.y, cs[k], s1);
        }
        reinterpret_cast<double2 *>(out)[i] = make_double2(s0, s1);
    }
    if ((n & 1) && bx == 0 && threadIdx.x == 0) {
        double s = 0;
        for (int k = 0; k < K; ++k) s = rfma(V[k * ldv + n - 1], cs[k], s);
        out[n - 1] = s;
    }
}
__global__ void __launch_bounds__(KR_THREADS)
k_lincomb_dyn(const double *__restrict__ V, size_t ldv, const int *countp, const double *__restrict__ c,
              double *__restrict__ out, long long n) {
    lincomb_dyn_body(blockIdx.x, gridDim.x, V, ldv, countp, c, out, n);
}

}  // namespace dgh
