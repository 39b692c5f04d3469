// Batched dense LU with row partial pivoting (the first largest |a| wins ties, as LAPACK's
// getrf and Eigen's PartialPivLU choose), the block solves, and a multi-RHS back substitution.
//
// Matrices are row-major with row length ld >= m.  Columns m..ld-1 (an augmented right-hand
// side [B r] for the HDG condensation) receive the row swaps and the forward elimination, so
// after k_lu they hold L^{-1} P [B r]; k_backsolve then overwrites them with U^{-1} of that.
// One CTA factors one matrix at a time in a persistent loop over the batch; the panel of NB
// columns is factored in shared memory and the trailing matrix is updated in global memory
// (resident in L2 for the block being factored).
#pragma once
#include "dgh_common.cuh"

namespace dgh {

template <typename T> __device__ inline T tabs(T x) { return x < T(0) ? -x : x; }

constexpr int LU_THREADS = 256;

template <typename T, int NB, int TC>
constexpr size_t lu_smem_bytes(int m) {
    return sizeof(T) * ((size_t)m * (NB + 1) + (size_t)NB * TC) + sizeof(int) * ((size_t)m + NB);
}

template <typename T, int NB, int TC>
__global__ void __launch_bounds__(LU_THREADS)
k_lu(T *__restrict__ pool, size_t stride, int m, int ld, int count, int *__restrict__ perm_out, int *status,
     int singular_bit) {
    constexpr int PP = NB + 1;
    extern __shared__ __align__(16) unsigned char smraw[];
    T *P = reinterpret_cast<T *>(smraw);  // panel rows k0..m-1, NB columns, pitch PP
    T *U = P + (size_t)m * PP;            // U12 tile: NB x TC
    int *piv = reinterpret_cast<int *>(U + NB * TC);
    int *swp = piv + m;
    __shared__ T red_v[LU_THREADS / 32];
    __shared__ int red_i[LU_THREADS / 32];
    __shared__ int bad;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    for (int blk = blockIdx.x; blk < count; blk += gridDim.x) {
        T *A = pool + (size_t)blk * stride;
        for (int i = tid; i < m; i += LU_THREADS) piv[i] = i;
        if (tid == 0) bad = 0;
        __syncthreads();
        for (int k0 = 0; k0 < m; k0 += NB) {
            const int nb = min(NB, m - k0), rows = m - k0;
            for (int idx = tid; idx < rows * nb; idx += LU_THREADS) {
                const int r = idx / nb, c = idx % nb;
                P[r * PP + c] = A[(size_t)(k0 + r) * ld + k0 + c];
            }
            __syncthreads();
            // ---- unblocked factorisation of the panel
            for (int jj = 0; jj < nb; ++jj) {
                T best = T(-1);
                int bi = 0x7fffffff;
                for (int r = jj + tid; r < rows; r += LU_THREADS) {
                    const T a = tabs(P[r * PP + jj]);
                    if (a > best || (a == best && r < bi)) { best = a; bi = r; }
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const T ob = __shfl_down_sync(0xffffffffu, best, o);
                    const int oi = __shfl_down_sync(0xffffffffu, bi, o);
                    if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
                }
                if (lane == 0) { red_v[warp] = best; red_i[warp] = bi; }
                __syncthreads();
                if (tid == 0) {
                    T b0 = red_v[0];
                    int i0 = red_i[0];
                    for (int w = 1; w < LU_THREADS / 32; ++w)
                        if (red_v[w] > b0 || (red_v[w] == b0 && red_i[w] < i0)) { b0 = red_v[w]; i0 = red_i[w]; }
                    if (i0 == 0x7fffffff || !(b0 == b0)) i0 = jj;  // NaN column: keep the diagonal
                    swp[jj] = i0;
                }
                __syncthreads();
                const int p = swp[jj];
                if (p != jj)
                    for (int c = tid; c < nb; c += LU_THREADS) {
                        const T t = P[jj * PP + c];
                        P[jj * PP + c] = P[p * PP + c];
                        P[p * PP + c] = t;
                    }
                __syncthreads();
                const T pivot = P[jj * PP + jj];
                for (int r = jj + 1 + tid; r < rows; r += LU_THREADS) {
                    T l = P[r * PP + jj];
                    if (pivot != T(0)) l = l / pivot;
                    P[r * PP + jj] = l;
                    for (int c = jj + 1; c < nb; ++c) P[r * PP + c] -= l * P[jj * PP + c];
                }
                __syncthreads();
            }
            // ---- write the panel back
            for (int idx = tid; idx < rows * nb; idx += LU_THREADS) {
                const int r = idx / nb, c = idx % nb;
                A[(size_t)(k0 + r) * ld + k0 + c] = P[r * PP + c];
            }
            // ---- apply the panel's row interchanges to all other columns, in order
            for (int jj = 0; jj < nb; ++jj) {
                const int r1 = k0 + jj, r2 = k0 + swp[jj];
                if (r1 != r2) {
                    for (int c = tid; c < ld - nb; c += LU_THREADS) {
                        const int col = c < k0 ? c : c + nb;
                        const T t = A[(size_t)r1 * ld + col];
                        A[(size_t)r1 * ld + col] = A[(size_t)r2 * ld + col];
                        A[(size_t)r2 * ld + col] = t;
                    }
                    if (tid == 0) {
                        const int t = piv[r1];
                        piv[r1] = piv[r2];
                        piv[r2] = t;
                    }
                }
                __syncthreads();
            }
            // ---- U12 = L11^{-1} A12 and the trailing update, one column tile at a time
            for (int c0 = k0 + nb; c0 < ld; c0 += TC) {
                const int tc = min(TC, ld - c0);
                for (int idx = tid; idx < nb * TC; idx += LU_THREADS) {
                    const int i = idx / TC, c = idx % TC;
                    U[i * TC + c] = c < tc ? A[(size_t)(k0 + i) * ld + c0 + c] : T(0);
                }
                __syncthreads();
                if (tid < tc)
                    for (int i = 1; i < nb; ++i) {
                        T val = U[i * TC + tid];
                        for (int l = 0; l < i; ++l) val -= P[i * PP + l] * U[l * TC + tid];
                        U[i * TC + tid] = val;
                    }
                __syncthreads();
                for (int idx = tid; idx < nb * tc; idx += LU_THREADS) {
                    const int i = idx / tc, c = idx % tc;
                    A[(size_t)(k0 + i) * ld + c0 + c] = U[i * TC + c];
                }
                // trailing rows k0+nb .. m-1
                const int R = rows - nb;
                const int tx = tid % (TC / 4), ty = tid / (TC / 4);
                constexpr int TY = LU_THREADS / (TC / 4);
                for (int rb = 0; rb < R; rb += 4 * TY) {
                    T acc[4][4];
                    int rr[4];
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        rr[k] = rb + ty + TY * k;
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const int c = 4 * tx + j;
                            acc[k][j] = (rr[k] < R && c < tc) ? A[(size_t)(k0 + nb + rr[k]) * ld + c0 + c] : T(0);
                        }
                    }
                    for (int l = 0; l < nb; ++l) {
                        T uu[4];
#pragma unroll
                        for (int j = 0; j < 4; ++j) uu[j] = U[l * TC + 4 * tx + j];
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const T lv = rr[k] < R ? P[(nb + rr[k]) * PP + l] : T(0);
#pragma unroll
                            for (int j = 0; j < 4; ++j) acc[k][j] -= lv * uu[j];
                        }
                    }
#pragma unroll
                    for (int k = 0; k < 4; ++k)
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const int c = 4 * tx + j;
                            if (rr[k] < R && c < tc) A[(size_t)(k0 + nb + rr[k]) * ld + c0 + c] = acc[k][j];
                        }
                }
                __syncthreads();
            }
        }
        // ---- singularity check on the diagonal (block_jacobi.hpp:16-18, dense_lu.hpp:13-16)
        for (int i = tid; i < m; i += LU_THREADS) {
            const T d = A[(size_t)i * ld + i];
            const double dd = (double)d;
            if (!isfinite(dd) || !(fabs(dd) > 2.2250738585072014e-308)) bad = 1;
            perm_out[(size_t)blk * m + i] = piv[i];
        }
        __syncthreads();
        if (tid == 0 && bad) atomicOr(status, singular_bit);
        __syncthreads();
    }
}

// Block solve z = A^{-1} b with the factors of k_lu (block_jacobi.hpp:24-39): permute, unit
// lower solve, upper solve.  Rows are streamed once; 32-row tiles use a warp-per-row GEMV
// against the solved part and a one-warp triangular solve for the diagonal tile.  T is the
// factor and arithmetic precision; b and z are FP64.
template <typename T>
__global__ void __launch_bounds__(LU_THREADS)
k_lu_solve(const T *__restrict__ pool, const int *__restrict__ perm, size_t stride, int m, int count,
           const double *__restrict__ rhs, double *__restrict__ z) {
    extern __shared__ __align__(16) unsigned char smraw[];
    T *y = reinterpret_cast<T *>(smraw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = LU_THREADS / 32;
    for (int blk = blockIdx.x; blk < count; blk += gridDim.x) {
        const T *A = pool + (size_t)blk * stride;
        const int *pm = perm + (size_t)blk * m;
        const double *b = rhs + (size_t)blk * m;
        for (int i = tid; i < m; i += LU_THREADS) y[i] = (T)b[pm[i]];
        __syncthreads();
        // forward: L y = P b (unit diagonal)
        for (int r0 = 0; r0 < m; r0 += 32) {
            const int nt = min(32, m - r0);
            if (r0 > 0) {
                for (int rr = warp; rr < nt; rr += NW) {
                    const T *row = A + (size_t)(r0 + rr) * m;
                    T s = 0;
                    for (int j = lane; j < r0; j += 32) s += row[j] * y[j];
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
                    if (lane == 0) y[r0 + rr] -= s;
                }
                __syncthreads();
            }
            if (warp == 0) {
                T yi = lane < nt ? y[r0 + lane] : T(0);
                T L[32];
                const T *row = A + (size_t)(r0 + min(lane, nt - 1)) * m + r0;
#pragma unroll
                for (int j = 0; j < 32; ++j) L[j] = (j < lane && lane < nt) ? row[j] : T(0);
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const T yj = __shfl_sync(0xffffffffu, yi, j);
                    if (j < nt) yi -= L[j] * yj;
                }
                if (lane < nt) y[r0 + lane] = yi;
            }
            __syncthreads();
        }
        // backward: U z = y
        const int last = ((m - 1) / 32) * 32;
        for (int r0 = last; r0 >= 0; r0 -= 32) {
            const int nt = min(32, m - r0), hi = r0 + nt;
            if (hi < m) {
                for (int rr = warp; rr < nt; rr += NW) {
                    const T *row = A + (size_t)(r0 + rr) * m;
                    T s = 0;
                    for (int j = hi + lane; j < m; j += 32) s += row[j] * y[j];
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
                    if (lane == 0) y[r0 + rr] -= s;
                }
                __syncthreads();
            }
            if (warp == 0) {
                T yi = lane < nt ? y[r0 + lane] : T(0);
                T Ur[32];
                const T *row = A + (size_t)(r0 + min(lane, nt - 1)) * m + r0;
#pragma unroll
                for (int j = 0; j < 32; ++j) Ur[j] = (j >= lane && j < nt && lane < nt) ? row[j] : T(0);
#pragma unroll
                for (int j = 31; j >= 0; --j) {
                    if (j < nt) {
                        if (lane == j) yi = yi / Ur[j];
                        const T yj = __shfl_sync(0xffffffffu, yi, j);
                        if (lane < j) yi -= Ur[j] * yj;
                    }
                }
                if (lane < nt) y[r0 + lane] = yi;
            }
            __syncthreads();
        }
        for (int i = tid; i < m; i += LU_THREADS) z[(size_t)blk * m + i] = (double)y[i];
        __syncthreads();
    }
}

// Multi-RHS back substitution U X = Y in place on columns [m, ld) of each factored matrix.
// Row tiles of 32 from the bottom; RHS tiles of 64 columns.  Per tile: Y_I -= U_{I,>I} X_{>I}
// staged through shared memory in chunks of 32, then a column-parallel 32x32 triangular solve.
template <typename T>
__global__ void __launch_bounds__(LU_THREADS)
k_backsolve(T *__restrict__ pool, size_t stride, int m, int ld, int count) {
    constexpr int RT = 32, CT = 64, KC = 16;
    __shared__ T Us[RT][KC + 1];
    __shared__ T Xk[KC][CT];
    __shared__ T Xs[RT][CT + 1];
    __shared__ T Ud[RT][RT + 1];
    const int tid = threadIdx.x, tx = tid % 32, ty = tid / 32;  // 8 x 32
    const int nrhs = ld - m;
    for (int blk = blockIdx.x; blk < count; blk += gridDim.x) {
        T *A = pool + (size_t)blk * stride;
        for (int cb = 0; cb < nrhs; cb += CT) {
            const int ct = min(CT, nrhs - cb);
            const int last = ((m - 1) / RT) * RT;
            for (int r0 = last; r0 >= 0; r0 -= RT) {
                const int nt = min(RT, m - r0), hi = r0 + nt;
                T acc[4][2];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int r = ty + 8 * k;
#pragma unroll
                    for (int j = 0; j < 2; ++j) {
                        const int c = tx + 32 * j;
                        acc[k][j] = (r < nt && c < ct) ? A[(size_t)(r0 + r) * ld + m + cb + c] : T(0);
                    }
                }
                for (int l0 = hi; l0 < m; l0 += KC) {
                    const int kc = min(KC, m - l0);
                    for (int idx = tid; idx < RT * KC; idx += LU_THREADS) {
                        const int r = idx / KC, l = idx % KC;
                        Us[r][l] = (r < nt && l < kc) ? A[(size_t)(r0 + r) * ld + l0 + l] : T(0);
                    }
                    for (int idx = tid; idx < KC * CT; idx += LU_THREADS) {
                        const int l = idx / CT, c = idx % CT;
                        Xk[l][c] = (l < kc && c < ct) ? A[(size_t)(l0 + l) * ld + m + cb + c] : T(0);
                    }
                    __syncthreads();
                    for (int l = 0; l < kc; ++l) {
                        const T x0 = Xk[l][tx], x1 = Xk[l][tx + 32];
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const T u = Us[ty + 8 * k][l];
                            acc[k][0] -= u * x0;
                            acc[k][1] -= u * x1;
                        }
                    }
                    __syncthreads();
                }
#pragma unroll
                for (int k = 0; k < 4; ++k)
#pragma unroll
                    for (int j = 0; j < 2; ++j) Xs[ty + 8 * k][tx + 32 * j] = acc[k][j];
                for (int idx = tid; idx < RT * RT; idx += LU_THREADS) {
                    const int r = idx / RT, c = idx % RT;
                    Ud[r][c] = (r < nt && c < nt) ? A[(size_t)(r0 + r) * ld + r0 + c] : T(0);
                }
                __syncthreads();
                if (tid < ct)
                    for (int i = nt - 1; i >= 0; --i) {
                        T val = Xs[i][tid];
                        for (int l = i + 1; l < nt; ++l) val -= Ud[i][l] * Xs[l][tid];
                        Xs[i][tid] = val / Ud[i][i];
                    }
                __syncthreads();
                for (int idx = tid; idx < nt * ct; idx += LU_THREADS) {
                    const int r = idx / ct, c = idx % ct;
                    A[(size_t)(r0 + r) * ld + m + cb + c] = Xs[r][c];
                }
                __syncthreads();
            }
        }
    }
}

}  // namespace dgh
