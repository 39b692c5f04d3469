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

#include <cuda_fp16.h>

namespace dgh {

template <typename T> __device__ inline T tabs(T x) { return x < T(0) ? -x : x; }

// Slab layout of a factored block (written by k_lu with slab_out, read by k_lu_solve): rows
// 32s..32s+nt-1 form slab s; inside a slab, columns come in groups of W = 16 bytes / sizeof(T)
// and each row's W values of a group are adjacent: element (32s + i, j) sits at
// 32 s m + (j / W) nt W + i W + j % W.  Lane i of a warp then loads its row's next W columns as
// one 16-byte vector, and the warp's load of a column group is nt*16 contiguous bytes.
// m = 4n^2 (cells) and 4n (faces) are multiples of W, so every group is complete.
template <typename T> struct SlabVec;
template <> struct SlabVec<double> {
    using V = double2;
    static constexpr int W = 2;
    __device__ static double dot(const V &a, const double *y) { return a.x * y[0] + a.y * y[1]; }
    __device__ static double dotv(const V &a, const V &y) { return a.x * y.x + a.y * y.y; }
};
template <> struct SlabVec<float> {
    using V = float4;
    static constexpr int W = 4;
    __device__ static float dot(const V &a, const float *y) { return a.x * y[0] + a.y * y[1] + a.z * y[2] + a.w * y[3]; }
    __device__ static float dotv(const V &a, const V &y) { return a.x * y.x + a.y * y.y + a.z * y.z + a.w * y.w; }
};
template <typename T> __device__ inline size_t slab_at(int nt, int i, int j) {
    constexpr int W = SlabVec<T>::W;
    return (size_t)(j / W) * nt * W + i * W + j % W;
}

constexpr int LU_THREADS = 256;

template <typename T, int NB, int TC>
constexpr size_t lu_smem_bytes(int m) {
    return sizeof(T) * ((size_t)m * (NB + 1) + (size_t)NB * TC + (size_t)NB * (NB + 1)) +
           sizeof(int) * ((size_t)4 * m + NB);
}

// Unblocked LU of the NB-column panel held in shared memory by the whole CTA: per column, a
// warp-shuffle pivot search (the first largest |a| wins) whose per-warp candidates every thread
// combines in the same order, the row interchange, and the rank-1 update with threads owning
// rows (three barriers per column).  The interchanges go to swp[] (panel-relative).  Also forms
// Li = L11^{-1}, the inverse of the unit-lower diagonal block, so U12 = L11^{-1} A12 is a product.
template <typename T, int NB>
__device__ void panel_factor(T *P, int rows, int nb, int *swp, T *Li, T *cand_v, int *cand_i) {
    constexpr int PP = NB + 1, NW = LU_THREADS / 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int jj = 0; jj < nb; ++jj) {
        T best = T(-1);
        int bi = 0x7fffffff;
        for (int r = jj + tid; r < rows; r += LU_THREADS) {
            const T a = tabs(P[r * PP + jj]);
            if (a > best) { best = a; bi = r; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const T ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
        }
        if (lane == 0) {
            cand_v[warp] = best;
            cand_i[warp] = bi;
        }
        __syncthreads();
        best = cand_v[0];
        bi = cand_i[0];
#pragma unroll
        for (int w = 1; w < NW; ++w)
            if (cand_v[w] > best || (cand_v[w] == best && cand_i[w] < bi)) { best = cand_v[w]; bi = cand_i[w]; }
        const int p = (bi == 0x7fffffff || !(best == best)) ? jj : bi;  // NaN column: keep the diagonal
        if (tid == 0) swp[jj] = p;
        if (p != jj && tid < nb) {
            const T t = P[jj * PP + tid];
            P[jj * PP + tid] = P[p * PP + tid];
            P[p * PP + tid] = t;
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
    if (tid < nb) {  // Li = L11^{-1}, column tid
        const int c = tid;
        for (int i = 0; i < nb; ++i) Li[i * PP + c] = i == c ? T(1) : T(0);
        for (int i = c + 1; i < nb; ++i) {
            T s = 0;
            for (int l = c; l < i; ++l) s += P[i * PP + l] * Li[l * PP + c];
            Li[i * PP + c] = -s;
        }
    }
    __syncthreads();
}

// Trailing update of one column tile with FFMA register tiles: each thread owns 4 rows x 4
// columns, the rows one pass ahead in registers (FP32 factors).
template <typename T, int NB, int TC>
__device__ __forceinline__ void trailing_ffma(T *__restrict__ A, int ld, int k0, int nb, int R, int c0, int tc,
                                              const int *src, const T *P, const T *U) {
    constexpr int PP = NB + 1;
    const int tid = threadIdx.x;
    const int tx = tid % (TC / 4), ty = tid / (TC / 4);
    constexpr int TY = LU_THREADS / (TC / 4);
    T nxt[4][4];
    auto load_pass = [&](int rb) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int r = min(rb + ty + TY * k, R - 1);
            const T *rowp = A + (size_t)(k0 + src[nb + r]) * ld + c0 + 4 * tx;
#pragma unroll
            for (int j = 0; j < 4; ++j) nxt[k][j] = (4 * tx + j < tc) ? rowp[j] : T(0);
        }
    };
    if (R > 0) load_pass(0);
    for (int rb = 0; rb < R; rb += 4 * TY) {
        T acc[4][4];
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[k][j] = nxt[k][j];
        if (rb + 4 * TY < R) load_pass(rb + 4 * TY);
        const T *lrow[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) lrow[k] = P + (size_t)(nb + min(rb + ty + TY * k, R - 1)) * PP;
        const T *ucol = U + 4 * tx;
#pragma unroll 4
        for (int l = 0; l < nb; ++l) {
            T uu[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) uu[j] = ucol[l * TC + j];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const T lv = lrow[k][l];
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[k][j] -= lv * uu[j];
            }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int r = rb + ty + TY * k;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = 4 * tx + j;
                if (r < R && c < tc) A[(size_t)(k0 + nb + r) * ld + c0 + c] = acc[k][j];
            }
        }
    }
}

// FP64 DMMA m8n8k4: d = a b + d on one 8x8 tile, a the 8x4 and b the 4x8 operand fragment
// (lane l holds a[l/4][l%4], b[l%4][l/4] and d[l/4][2(l%4) .. 2(l%4)+1]).
__device__ __forceinline__ void dmma8x8x4(double (&d)[2], double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// Trailing update of one 32-column tile on the FP64 tensor pipe: each warp owns 32 rows x 32
// columns (4 x 4 DMMA tiles, 32 accumulators per lane), loads its rows through the panel's
// gather src[], runs nb/4 k-steps against -L21 (shared panel) and U12 (shared tile), and
// stores the updated rows in place.
template <int NB>
__device__ __forceinline__ void trailing_dmma(double *__restrict__ A, int ld, int k0, int nb, int R, int c0, int tc,
                                              const int *src, const double *P, const double *U) {
    constexpr int PP = NB + 1, TC = 32, NW = LU_THREADS / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int lr = lane >> 2, lc = lane & 3;
    for (int rb = warp * 32; rb < R; rb += NW * 32) {
        double c[4][4][2];
        int srow[4];
        bool valid[4];
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) {
            const int r = rb + mt * 8 + lr;
            valid[mt] = r < R;
            srow[mt] = valid[mt] ? k0 + src[nb + r] : 0;
        }
#pragma unroll
        for (int mt = 0; mt < 4; ++mt)
#pragma unroll
            for (int nt = 0; nt < 4; ++nt)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int col = nt * 8 + 2 * lc + e;
                    c[mt][nt][e] = (valid[mt] && col < tc) ? A[(size_t)srow[mt] * ld + c0 + col] : 0.;
                }
        for (int kk = 0; kk < nb; kk += 4) {
            double a[4], b[4];
#pragma unroll
            for (int mt = 0; mt < 4; ++mt) {
                const int r = rb + mt * 8 + lr;
                a[mt] = valid[mt] ? -P[(size_t)(nb + r) * PP + kk + lc] : 0.;
            }
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) b[nt] = U[(kk + lc) * TC + nt * 8 + lr];
#pragma unroll
            for (int mt = 0; mt < 4; ++mt)
#pragma unroll
                for (int nt = 0; nt < 4; ++nt) dmma8x8x4(c[mt][nt], a[mt], b[nt]);
        }
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) {
            if (!valid[mt]) continue;
            double *row = A + (size_t)(k0 + nb + rb + mt * 8 + lr) * ld + c0;
#pragma unroll
            for (int nt = 0; nt < 4; ++nt)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int col = nt * 8 + 2 * lc + e;
                    if (col < tc) row[col] = c[mt][nt][e];
                }
        }
    }
}

// Right-looking blocked LU.  Row interchanges are never executed one at a time: the columns
// right of the panel are read through the panel's row permutation when its U12 tile and the
// trailing rows are formed (a row moved by the panel's pivoting comes from the panel's top
// rows, which are written only after the trailing update, so the gather is race-free), and the
// L columns of earlier panels are permuted once at the end (the L fix-up, flag bit 1; the FP64
// augmented HDG matrices skip it, as their L factor is not needed after the forward
// elimination, while the FP32 condensation keeps its factors for later solves).  Flag bit 0
// converts the factored block in place to the slab layout of k_lu_solve (ld == m only).
template <typename T, int NB, int TC>
__global__ void __launch_bounds__(LU_THREADS)
k_lu(T *__restrict__ pool, size_t stride, int m, int ld, int count, int *__restrict__ perm_out, int *status,
     int singular_bit, int flags) {
    constexpr int PP = NB + 1;
    static_assert(LU_THREADS % TC == 0 && NB % (LU_THREADS / TC) == 0, "tile shape");
    extern __shared__ __align__(16) unsigned char smraw[];
    T *P = reinterpret_cast<T *>(smraw);  // panel rows k0..m-1, NB columns, pitch PP
    T *U = P + (size_t)m * PP;            // A12 / U12 tile: NB x TC
    T *Li = U + NB * TC;                  // L11^{-1}: NB x NB, pitch PP
    int *piv = reinterpret_cast<int *>(Li + NB * PP);  // position -> original row
    int *src = piv + m;                   // panel-relative source position of each position
    int *ipiv = src + m;                  // LAPACK-style interchange list
    int *inv = ipiv + m;                  // scratch for the L fix-up
    int *swp = inv + m;
    __shared__ int bad;
    __shared__ T cand_v[LU_THREADS / 32];
    __shared__ int cand_i[LU_THREADS / 32];
    static_assert(NB == 32, "panel rows are moved by one warp lane per column");
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = LU_THREADS / 32;

    for (int blk = blockIdx.x; blk < count; blk += gridDim.x) {
        T *A = pool + (size_t)blk * stride;
        for (int i = tid; i < m; i += LU_THREADS) piv[i] = i;
        if (tid == 0) bad = 0;
        __syncthreads();
        for (int k0 = 0; k0 < m; k0 += NB) {
            const int nb = min(NB, m - k0), rows = m - k0;
            if (lane < nb)
                for (int r = warp; r < rows; r += NW) P[r * PP + lane] = A[(size_t)(k0 + r) * ld + k0 + lane];
            for (int i = tid; i < rows; i += LU_THREADS) src[i] = i;
            __syncthreads();
            panel_factor<T, NB>(P, rows, nb, swp, Li, cand_v, cand_i);
            if (tid == 0)
                for (int jj = 0; jj < nb; ++jj) {
                    const int p = swp[jj];
                    ipiv[k0 + jj] = k0 + p;
                    int t = src[jj]; src[jj] = src[p]; src[p] = t;
                    t = piv[k0 + jj]; piv[k0 + jj] = piv[k0 + p]; piv[k0 + p] = t;
                }
            if (lane < nb)
                for (int r = warp; r < rows; r += NW) A[(size_t)(k0 + r) * ld + k0 + lane] = P[r * PP + lane];
            __syncthreads();
            for (int c0 = k0 + nb; c0 < ld; c0 += TC) {
                const int tc = min(TC, ld - c0);
                for (int idx = tid; idx < NB * TC; idx += LU_THREADS) {
                    const int i = idx / TC, c = idx % TC;
                    U[i * TC + c] = (c < tc && i < nb) ? A[(size_t)(k0 + src[i]) * ld + c0 + c] : T(0);
                }
                __syncthreads();
                {  // U12 = L11^{-1} A12
                    constexpr int RG = LU_THREADS / TC, RPT = NB / RG;
                    const int c = tid % TC, rg = tid / TC;
                    T out[RPT];
#pragma unroll
                    for (int q = 0; q < RPT; ++q) {
                        const int i = rg + RG * q;
                        T acc = 0;
                        for (int l = 0; l <= i && l < nb; ++l) acc += Li[i * PP + l] * U[l * TC + c];
                        out[q] = acc;
                    }
                    __syncthreads();
#pragma unroll
                    for (int q = 0; q < RPT; ++q) U[(rg + RG * q) * TC + c] = out[q];
                }
                __syncthreads();
                // trailing rows: A[k0+nb+r] = A[k0+src[nb+r]] - L21 U12
                if constexpr (sizeof(T) == 8 && TC == 32) trailing_dmma<NB>(A, ld, k0, nb, rows - nb, c0, tc, src, P, U);
                else trailing_ffma<T, NB, TC>(A, ld, k0, nb, rows - nb, c0, tc, src, P, U);
                __syncthreads();
                for (int i = tid / TC; i < nb; i += LU_THREADS / TC) {
                    const int c = tid % TC;
                    if (c < tc) A[(size_t)(k0 + i) * ld + c0 + c] = U[i * TC + c];
                }
                __syncthreads();
            }
        }
        // ---- L fix-up: panel q's L rows were written in the arrangement after panel q; gather
        // them into the final arrangement (piv) through the inverse arrangement of that time.
        if (flags & 2) {
            for (int i = tid; i < m; i += LU_THREADS) {
                src[i] = i;  // arrangement: position -> original row
                inv[i] = i;  // original row -> position
            }
            __syncthreads();
            for (int k0 = 0; k0 < m; k0 += NB) {
                const int nb = min(NB, m - k0), base = k0 + nb;
                if (tid == 0)
                    for (int jj = 0; jj < nb; ++jj) {
                        const int a = k0 + jj, b = ipiv[k0 + jj];
                        const int ra = src[a], rb = src[b];
                        src[a] = rb; src[b] = ra;
                        inv[rb] = a; inv[ra] = b;
                    }
                __syncthreads();
                if (base < m && lane < nb) {
                    for (int i = warp; i < m - base; i += NW) P[i * PP + lane] = A[(size_t)inv[piv[base + i]] * ld + k0 + lane];
                }
                __syncthreads();
                if (base < m && lane < nb) {
                    for (int i = warp; i < m - base; i += NW) A[(size_t)(base + i) * ld + k0 + lane] = P[i * PP + lane];
                }
                __syncthreads();
            }
        }
        // ---- singularity check on the diagonal (block_jacobi.hpp:16-18, dense_lu.hpp:13-16)
        for (int i = tid; i < m; i += LU_THREADS) {
            const double dd = (double)A[(size_t)i * ld + i];
            if (!isfinite(dd) || !(fabs(dd) > 2.2250738585072014e-308)) bad = 1;
            perm_out[(size_t)blk * m + i] = piv[i];
        }
        __syncthreads();
        if (tid == 0 && bad) atomicOr(status, singular_bit);
        // ---- in-place conversion to the slab layout read by k_lu_solve (ld == m only)
        if (flags & 1) {
            constexpr int W = SlabVec<T>::W;
            for (int r0 = 0; r0 < m; r0 += 32) {
                const int nt = min(32, m - r0);
                T *reg = A + (size_t)r0 * m;
                for (int idx = tid; idx < nt * m; idx += LU_THREADS) P[idx] = reg[idx];
                __syncthreads();
                // destination index e = g*nt*W + i*W + w holds row i, column g*W + w
                for (int g = warp; g < m / W; g += NW)
                    for (int e = lane; e < nt * W; e += 32) reg[(size_t)g * nt * W + e] = P[(e / W) * m + g * W + e % W];
                __syncthreads();
            }
        }
        __syncthreads();
    }
}

// LU with row partial pivoting of narrow blocks (m <= 64, ld == m: the HDG face blocks, m = 4n)
// with one warp per block in shared memory, written out in the slab layout of k_lu_solve.  The
// pivot rule and the singularity test are k_lu's (first largest |a|; a NaN column keeps its
// diagonal; a non-finite or subnormal-or-zero U diagonal sets singular_bit); lane r owns rows r
// and r + 32 and eliminates them column by column.  Shared memory per warp: m (m + 1) T.
constexpr int NARROW_THREADS = 128;
template <typename T> constexpr size_t lu_narrow_smem_bytes(int m) {
    return (size_t)(NARROW_THREADS / 32) * m * (m + 1) * sizeof(T);
}
template <typename T>
__global__ void __launch_bounds__(NARROW_THREADS)
k_lu_narrow(T *__restrict__ pool, int m, int count, int *__restrict__ perm_out, int *status, int singular_bit) {
    constexpr int W = SlabVec<T>::W;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, pitch = m + 1;
    T *S = reinterpret_cast<T *>(smraw) + (size_t)wib * m * pitch;
    const int warps = gridDim.x * (NARROW_THREADS / 32);
    for (int blk = blockIdx.x * (NARROW_THREADS / 32) + wib; blk < count; blk += warps) {
        T *A = pool + (size_t)blk * m * m;
        for (int e = lane; e < m * m; e += 32) S[(e / m) * pitch + e % m] = A[e];
        int orig0 = lane, orig1 = lane + 32;  // original rows now at positions lane, lane + 32
        __syncwarp();
        for (int j = 0; j < m; ++j) {
            T best = T(-1);
            int bi = 0x7fffffff;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = lane + 32 * h;
                if (r >= j && r < m) {
                    const T a = tabs(S[r * pitch + j]);
                    if (a > best) { best = a; bi = r; }
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const T ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
            }
            const int p = (bi == 0x7fffffff || !(best == best)) ? j : bi;
            if (p != j) {
                for (int c = lane; c < m; c += 32) {
                    const T t = S[j * pitch + c];
                    S[j * pitch + c] = S[p * pitch + c];
                    S[p * pitch + c] = t;
                }
                // the original row indices follow the rows
                const int oj = __shfl_sync(0xffffffffu, j < 32 ? orig0 : orig1, j & 31);
                const int op = __shfl_sync(0xffffffffu, p < 32 ? orig0 : orig1, p & 31);
                if (lane == (j & 31)) { if (j < 32) orig0 = op; else orig1 = op; }
                if (lane == (p & 31)) { if (p < 32) orig0 = oj; else orig1 = oj; }
            }
            __syncwarp();
            const T pivot = S[j * pitch + j];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = lane + 32 * h;
                if (r > j && r < m) {
                    T l = S[r * pitch + j];
                    if (pivot != T(0)) l = l / pivot;
                    S[r * pitch + j] = l;
                    for (int c = j + 1; c < m; ++c) S[r * pitch + c] -= l * S[j * pitch + c];
                }
            }
            __syncwarp();
        }
        bool bad = false;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = lane + 32 * h;
            if (r < m) {
                const double dd = (double)S[r * pitch + r];
                if (!isfinite(dd) || !(fabs(dd) > 2.2250738585072014e-308)) bad = true;
                perm_out[(size_t)blk * m + r] = h ? orig1 : orig0;
            }
        }
        if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(status, singular_bit);
        // slab layout: element (r, c) of slab s = r / 32 at 32 s m + (c / W) nt W + (r % 32) W + c % W
        for (int e = lane; e < m * m; e += 32) {
            const int s = e / (32 * m), off = e - s * 32 * m, nt = min(32, m - 32 * s);
            const int g = off / (nt * W), rem = off - g * nt * W, i = rem / W, w = rem % W;
            A[e] = S[(32 * s + i) * pitch + g * W + w];
        }
        __syncwarp();
    }
}

// Explicit inverses of narrow FP64 blocks (m <= 64, the HDG face blocks in the mixed form), one
// warp per block in shared memory: k_lu_narrow's pivoted LU (same pivot rule and singularity
// test), then A^{-1} = U^{-1} L^{-1} P column by column (lane c owns columns c and c + 32), written
// rounded to FP32 in groups of four columns (element (r, c) at (c / 4) 4m + 4r + c % 4, m a
// multiple of 4) so that k_inv_apply's lane r reads its row as 16-byte vectors.  Applying an
// FP32 inverse is a dense product with no dependent triangle steps, which for 36-wide blocks
// is what bounds the triangular solves.  Shared memory per warp: 2 m (m + 1) doubles.
constexpr int INV_THREADS = 128;
inline size_t inv_narrow_smem_bytes(int m) { return (size_t)(INV_THREADS / 32) * 2 * m * (m + 1) * sizeof(double); }
__global__ void __launch_bounds__(INV_THREADS)
k_inv_narrow(const double *__restrict__ pool, int m, int count, float *__restrict__ inv_out, int *status,
             int singular_bit) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, pitch = m + 1;
    double *S = reinterpret_cast<double *>(smraw) + (size_t)wib * 2 * m * pitch, *X = S + (size_t)m * pitch;
    const int warps = gridDim.x * (INV_THREADS / 32);
    for (int blk = blockIdx.x * (INV_THREADS / 32) + wib; blk < count; blk += warps) {
        const double *A = pool + (size_t)blk * m * m;
        for (int e = lane; e < m * m; e += 32) S[(e / m) * pitch + e % m] = A[e];
        int orig0 = lane, orig1 = lane + 32;
        __syncwarp();
        for (int j = 0; j < m; ++j) {
            double best = -1.;
            int bi = 0x7fffffff;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = lane + 32 * h;
                if (r >= j && r < m) {
                    const double a = fabs(S[r * pitch + j]);
                    if (a > best) { best = a; bi = r; }
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
            }
            const int p = (bi == 0x7fffffff || !(best == best)) ? j : bi;
            if (p != j) {
                for (int c = lane; c < m; c += 32) {
                    const double t = S[j * pitch + c];
                    S[j * pitch + c] = S[p * pitch + c];
                    S[p * pitch + c] = t;
                }
                const int oj = __shfl_sync(0xffffffffu, j < 32 ? orig0 : orig1, j & 31);
                const int op = __shfl_sync(0xffffffffu, p < 32 ? orig0 : orig1, p & 31);
                if (lane == (j & 31)) { if (j < 32) orig0 = op; else orig1 = op; }
                if (lane == (p & 31)) { if (p < 32) orig0 = oj; else orig1 = oj; }
            }
            __syncwarp();
            const double pivot = S[j * pitch + j];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = lane + 32 * h;
                if (r > j && r < m) {
                    double l = S[r * pitch + j];
                    if (pivot != 0.) l = l / pivot;
                    S[r * pitch + j] = l;
                    for (int c = j + 1; c < m; ++c) S[r * pitch + c] -= l * S[j * pitch + c];
                }
            }
            __syncwarp();
        }
        bool bad = false;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = lane + 32 * h;
            if (r < m) {
                const double dd = S[r * pitch + r];
                if (!isfinite(dd) || !(fabs(dd) > 2.2250738585072014e-308)) bad = true;
            }
        }
        if (__any_sync(0xffffffffu, bad)) {
            if (lane == 0) atomicOr(status, singular_bit);
            continue;
        }
        // column c of A^{-1}: the right-hand side P e_c is the unit vector at the position i
        // whose original row is c (orig(i) == c); unit-lower forward, then upper backward
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int c = lane + 32 * h;
            int at = -1;
            for (int i = 0; i < m; ++i) {
                const int oi = __shfl_sync(0xffffffffu, i < 32 ? orig0 : orig1, i & 31);
                if (oi == c) at = i;
            }
            if (c < m) {
                for (int i = 0; i < at; ++i) X[i * pitch + c] = 0.;  // above the unit entry
                for (int i = at; i < m; ++i) {
                    double v = i == at ? 1. : 0.;
                    for (int k = at; k < i; ++k) v -= S[i * pitch + k] * X[k * pitch + c];
                    X[i * pitch + c] = v;
                }
                for (int i = m - 1; i >= 0; --i) {
                    double v = X[i * pitch + c];
                    for (int k = i + 1; k < m; ++k) v -= S[i * pitch + k] * X[k * pitch + c];
                    X[i * pitch + c] = v / S[i * pitch + i];
                }
            }
        }
        __syncwarp();
        float *out = inv_out + (size_t)blk * m * m;
        for (int e = lane; e < m * m; e += 32) {
            const int g = e / (4 * m), r = (e / 4) % m, cc = 4 * g + e % 4;
            out[e] = (float)X[r * pitch + cc];
        }
        __syncwarp();
    }
}

// z = A^{-1} b per block with the FP32 inverses of k_inv_narrow: one warp per block, lane r
// computes rows r and r + 32 (FP32 accumulation) from 16-byte loads of its row, b broadcast by
// shuffles.  m is a multiple of 4 (m = 4n).
constexpr int INV_APPLY_THREADS = 256;
__device__ __forceinline__ void inv_apply_body(int bx, int G, const float *__restrict__ inv, int m, int count,
                                               const double *__restrict__ rhs, double *__restrict__ z) {
    const int lane = threadIdx.x & 31;
    const int warps = G * (INV_APPLY_THREADS / 32);
    for (int blk = bx * (INV_APPLY_THREADS / 32) + (threadIdx.x >> 5); blk < count; blk += warps) {
        const float4 *A4 = reinterpret_cast<const float4 *>(inv + (size_t)blk * m * m);
        const double *b = rhs + (size_t)blk * m;
        const float b0 = lane < m ? (float)b[lane] : 0.f, b1 = lane + 32 < m ? (float)b[lane + 32] : 0.f;
        float acc0 = 0.f, acc1 = 0.f;
        const bool r0 = lane < m, r1 = lane + 32 < m;
        const int groups = m / 4;
#pragma unroll 3
        for (int g = 0; g < groups; ++g) {
            float bj[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int j = 4 * g + e;
                bj[e] = j < 32 ? __shfl_sync(0xffffffffu, b0, j) : __shfl_sync(0xffffffffu, b1, j - 32);
            }
            if (r0) {
                const float4 a = A4[(size_t)g * m + lane];
                acc0 += a.x * bj[0] + a.y * bj[1] + a.z * bj[2] + a.w * bj[3];
            }
            if (r1) {
                const float4 a = A4[(size_t)g * m + lane + 32];
                acc1 += a.x * bj[0] + a.y * bj[1] + a.z * bj[2] + a.w * bj[3];
            }
        }
        if (r0) z[(size_t)blk * m + lane] = (double)acc0;
        if (r1) z[(size_t)blk * m + lane + 32] = (double)acc1;
    }
}
__global__ void __launch_bounds__(INV_APPLY_THREADS)
k_inv_apply(const float *__restrict__ inv, int m, int count, const double *__restrict__ rhs, double *__restrict__ z) {
    inv_apply_body(blockIdx.x, gridDim.x, inv, m, count, rhs, z);
}

// Block solve z = A^{-1} b with the factors of k_lu (block_jacobi.hpp:24-39): permute, unit
// lower solve, upper solve.  One warp owns one block and streams its factors exactly once with
// no CTA-wide barriers; lane i owns row 32 s + i of slab s and reads 16-byte column groups of
// the slab layout above.  Off-diagonal parts are per-lane dot products (four 16-byte loads in
// flight per lane, four accumulators); the diagonal triangles of the 32-row slabs are solved with
// warp shuffles.  T is the factor and arithmetic precision (FP32 factors accumulate in FP32);
// b and z are FP64.  The forward and backward sweeps share one loop body, which keeps the
// kernel at <= 48 registers (FP32; five 256-thread CTAs per SM) or 64 (FP64).  DIAG loads a full
// slab's diagonal row into registers before its triangle (all its loads in flight at once): the
// FP32 form for narrow blocks (the HDG face blocks, m = 4n), whose time is mostly triangles.
constexpr int SOLVE_THREADS = 256;
template <typename T, bool DIAG> constexpr int solve_min_blocks() { return sizeof(T) == 4 && !DIAG ? 5 : 4; }
// The body takes its block index bx and block count G explicitly (the batched solve of a
// lockstep batch runs it over each member's blocks).
template <typename T, bool DIAG>
__device__ __forceinline__ void lu_solve_body(int bx, int G, const T *__restrict__ pool, const int *__restrict__ perm,
                                              size_t stride, int m, int count, const double *__restrict__ rhs,
                                              double *__restrict__ z) {
    using SV = SlabVec<T>;
    using V = typename SV::V;
    constexpr int W = SV::W, ND = 32 / W;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    T *y = reinterpret_cast<T *>(smraw) + (size_t)wib * m;
    // m * sizeof(T) is a multiple of 16 (m = 4n^2 or 4n), so every warp's y is 16-byte aligned
    const V *yv = reinterpret_cast<const V *>(y);
    const int warps = G * (SOLVE_THREADS / 32);
    const int slabs = (m + 31) / 32;
    for (int blk = bx * (SOLVE_THREADS / 32) + wib; blk < count; blk += warps) {
        const T *A = pool + (size_t)blk * stride;
        const int *pm = perm + (size_t)blk * m;
        const double *b = rhs + (size_t)blk * m;
        for (int i = lane; i < m; i += 32) y[i] = (T)b[pm[i]];
        __syncwarp();
        // dir 0: forward, L y = P b (slabs in order, columns left of the slab); dir 1: backward,
        // U z = y (slabs in reverse, columns right of the slab)
        for (int dir = 0; dir < 2; ++dir) {
            for (int si = 0; si < slabs; ++si) {
                const int s = dir == 0 ? si : slabs - 1 - si;
                const int r0 = 32 * s, nt = min(32, m - r0), hi = r0 + nt;
                const T *S = A + (size_t)r0 * m;
                const V *Sv = reinterpret_cast<const V *>(S);
                const bool act = lane < nt;
                T acc0 = 0, acc1 = 0, acc2 = 0, acc3 = 0;
                if (act) {
                    const int g1 = dir == 0 ? r0 / W : m / W;
                    int g = dir == 0 ? 0 : hi / W;
                    for (; g + 4 <= g1; g += 4) {  // four independent 16-byte loads in flight per lane
                        const V a0 = Sv[(size_t)g * nt + lane], a1 = Sv[(size_t)(g + 1) * nt + lane];
                        const V a2 = Sv[(size_t)(g + 2) * nt + lane], a3 = Sv[(size_t)(g + 3) * nt + lane];
                        acc0 += SV::dotv(a0, yv[g]);
                        acc1 += SV::dotv(a1, yv[g + 1]);
                        acc2 += SV::dotv(a2, yv[g + 2]);
                        acc3 += SV::dotv(a3, yv[g + 3]);
                    }
                    for (; g < g1; ++g) acc0 += SV::dotv(Sv[(size_t)g * nt + lane], yv[g]);
                }
                T t = act ? y[r0 + lane] - ((acc0 + acc1) + (acc2 + acc3)) : T(0);
                if (DIAG && nt == 32) {
                    V d[ND];
#pragma unroll
                    for (int q = 0; q < ND; ++q) d[q] = Sv[(size_t)(r0 / W + q) * 32 + lane];
                    if (dir == 0) {
#pragma unroll
                        for (int q = 0; q < ND; ++q) {
                            const T *e = reinterpret_cast<const T *>(&d[q]);
#pragma unroll
                            for (int w = 0; w < W; ++w) {
                                const int jj = W * q + w;
                                const T l = lane > jj ? e[w] : T(0);
                                const T yj = __shfl_sync(0xffffffffu, t, jj);
                                t -= l * yj;
                            }
                        }
                    } else {
#pragma unroll
                        for (int q = ND - 1; q >= 0; --q) {
                            const T *e = reinterpret_cast<const T *>(&d[q]);
#pragma unroll
                            for (int w = W - 1; w >= 0; --w) {
                                const int jj = W * q + w;
                                const T u = e[w];
                                if (lane == jj) t = t / u;
                                const T yj = __shfl_sync(0xffffffffu, t, jj);
                                if (lane < jj) t -= u * yj;
                            }
                        }
                    }
                } else if (dir == 0) {
                    for (int jj = 0; jj < nt; ++jj) {
                        const T l = (act && lane > jj) ? S[slab_at<T>(nt, lane, r0 + jj)] : T(0);
                        const T yj = __shfl_sync(0xffffffffu, t, jj);
                        t -= l * yj;
                    }
                } else {
                    for (int jj = nt - 1; jj >= 0; --jj) {
                        // row `lane` uses U(lane, jj) only on and right of its diagonal: the
                        // lower half of the diagonal block was read by the forward sweep and is
                        // not fetched again
                        const T u = (act && lane <= jj) ? S[slab_at<T>(nt, lane, r0 + jj)] : T(1);
                        if (lane == jj) t = t / u;
                        const T yj = __shfl_sync(0xffffffffu, t, jj);
                        if (lane < jj) t -= u * yj;
                    }
                }
                if (act) y[r0 + lane] = t;
                __syncwarp();
            }
        }
        for (int i = lane; i < m; i += 32) z[(size_t)blk * m + i] = (double)y[i];
        __syncwarp();
    }
}
template <typename T, bool DIAG>
__global__ void __launch_bounds__(SOLVE_THREADS, (solve_min_blocks<T, DIAG>()))
k_lu_solve(const T *__restrict__ pool, const int *__restrict__ perm, size_t stride, int m, int count,
           const double *__restrict__ rhs, double *__restrict__ z) {
    lu_solve_body<T, DIAG>(blockIdx.x, gridDim.x, pool, perm, stride, m, count, rhs, z);
}

// ---- 16-bit factor storage (the DG cell blocks, DGH_PRECISION_MIXED16) -------------------------
// FP16 slabs with 8 columns per 16-byte group and rows padded to mp = m rounded up to 8 (zeros
// past column m): element (32 s + i, j) at 32 s mp + (j / 8) nt 8 + 8 i + j % 8.  The strictly
// lower part holds L (|L| <= 1 under partial pivoting); each row's upper part U(i, i..m-1) is
// stored divided by that row's largest |U(i, j)|, whose reciprocal is kept as an FP32 row scale,
// so every stored U row peaks at 1 and stays in FP16's normal range.
constexpr int H_W = 8;
__host__ __device__ constexpr int pad8(int m) { return (m + 7) / 8 * 8; }

// Packs row-major factored FP64 blocks (LU in place, row length m, rows in position order) into
// the FP16 slabs and row scales: one warp per 32-row slab of a block, lane i owning row 32 s + i.
__global__ void k_pack_half(const double *__restrict__ src, int m, int count, __half *__restrict__ dst,
                            float *__restrict__ row_scale) {
    const int mp = pad8(m), slabs = (m + 31) / 32, lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= (long long)count * slabs) return;
    const int blk = (int)(warp / slabs), s = (int)(warp % slabs), r0 = 32 * s, nt = min(32, m - r0);
    if (lane >= nt) return;
    const int row = r0 + lane;
    const double *ar = src + (size_t)blk * m * m + (size_t)row * m;
    __half *out = dst + (size_t)blk * m * mp + (size_t)r0 * mp;
    double big = 0;
    for (int j = row; j < m; ++j) big = fmax(big, fabs(ar[j]));
    const double inv = big > 0 ? 1. / big : 1.;
    row_scale[(size_t)blk * m + row] = (float)inv;
    for (int g = 0; g < mp / H_W; ++g) {
        __align__(16) __half v[H_W];
#pragma unroll
        for (int w = 0; w < H_W; ++w) {
            const int j = g * H_W + w;
            const double a = j < m ? ar[j] : 0.;
            v[w] = __double2half(j >= row ? a * inv : a);
        }
        *reinterpret_cast<uint4 *>(out + (size_t)g * nt * H_W + lane * H_W) = *reinterpret_cast<const uint4 *>(v);
    }
}

// z = A^{-1} b per block from the FP16 slabs: k_lu_solve's structure (one warp per block, lane
// i owns row 32 s + i, four 16-byte loads in flight, shuffled diagonal triangles) with FP32
// arithmetic; the backward sweep multiplies each row's right-hand side by its row scale.
__device__ __forceinline__ void lu_solve_half_body(int bx, int G, const __half *__restrict__ pool,
                                                   const float *__restrict__ row_scale, const int *__restrict__ perm,
                                                   int m, int count, const double *__restrict__ rhs,
                                                   double *__restrict__ z) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const int mp = pad8(m), lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    float *y = reinterpret_cast<float *>(smraw) + (size_t)wib * mp;
    const float4 *yv = reinterpret_cast<const float4 *>(y);
    const int warps = G * (SOLVE_THREADS / 32);
    const int slabs = (m + 31) / 32;
    auto dot8 = [&](const uint4 &a, int g) {
        const __half2 *h = reinterpret_cast<const __half2 *>(&a);
        const float4 y0 = yv[2 * g], y1 = yv[2 * g + 1];
        const float2 f0 = __half22float2(h[0]), f1 = __half22float2(h[1]);
        const float2 f2 = __half22float2(h[2]), f3 = __half22float2(h[3]);
        return (f0.x * y0.x + f0.y * y0.y) + (f1.x * y0.z + f1.y * y0.w) + (f2.x * y1.x + f2.y * y1.y) +
               (f3.x * y1.z + f3.y * y1.w);
    };
    for (int blk = bx * (SOLVE_THREADS / 32) + wib; blk < count; blk += warps) {
        const __half *A = pool + (size_t)blk * m * mp;
        const int *pm = perm + (size_t)blk * m;
        const float *rs = row_scale + (size_t)blk * m;
        const double *b = rhs + (size_t)blk * m;
        for (int i = lane; i < mp; i += 32) y[i] = i < m ? (float)b[pm[i]] : 0.f;
        __syncwarp();
        for (int dir = 0; dir < 2; ++dir) {
            for (int si = 0; si < slabs; ++si) {
                const int s = dir == 0 ? si : slabs - 1 - si;
                const int r0 = 32 * s, nt = min(32, m - r0), hi = r0 + nt;
                const __half *S = A + (size_t)r0 * mp;
                const uint4 *Sv = reinterpret_cast<const uint4 *>(S);
                const bool act = lane < nt;
                float acc0 = 0, acc1 = 0, acc2 = 0, acc3 = 0;
                if (act) {
                    // forward: the groups left of the slab; backward: the groups right of it (the
                    // last slab, whose end may fall inside a group, has none)
                    const int g1 = dir == 0 ? r0 / H_W : mp / H_W;
                    int g = dir == 0 ? 0 : (hi >= m ? mp / H_W : hi / H_W);
                    for (; g + 4 <= g1; g += 4) {
                        const uint4 a0 = Sv[(size_t)g * nt + lane], a1 = Sv[(size_t)(g + 1) * nt + lane];
                        const uint4 a2 = Sv[(size_t)(g + 2) * nt + lane], a3 = Sv[(size_t)(g + 3) * nt + lane];
                        acc0 += dot8(a0, g);
                        acc1 += dot8(a1, g + 1);
                        acc2 += dot8(a2, g + 2);
                        acc3 += dot8(a3, g + 3);
                    }
                    for (; g < g1; ++g) acc0 += dot8(Sv[(size_t)g * nt + lane], g);
                }
                // the slab's diagonal 32 x 32 block: this lane's row, four 16-byte groups loaded at
                // once (r0 is a multiple of 32, so the block starts a group)
                uint4 dg[4];
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    dg[q] = (act && 8 * q < nt) ? Sv[(size_t)(r0 / H_W + q) * nt + lane] : make_uint4(0, 0, 0, 0);
                float t = 0.f;
                if (act) t = (dir == 0 ? y[r0 + lane] : y[r0 + lane] * rs[r0 + lane]) - ((acc0 + acc1) + (acc2 + acc3));
                auto at = [&](int jj) {  // stored entry (row r0 + lane, column r0 + jj), jj a constant
                    const uint4 &v = dg[jj >> 3];
                    const int w = (jj >> 1) & 3;
                    const unsigned word = w == 0 ? v.x : w == 1 ? v.y : w == 2 ? v.z : v.w;
                    return __half2float(__ushort_as_half((unsigned short)((jj & 1) ? word >> 16 : word & 0xffffu)));
                };
                if (dir == 0) {
#pragma unroll
                    for (int jj = 0; jj < 32; ++jj) {
                        if (jj >= nt) break;
                        const float l = lane > jj ? at(jj) : 0.f;
                        const float yj = __shfl_sync(0xffffffffu, t, jj);
                        t -= l * yj;
                    }
                } else {
#pragma unroll
                    for (int jj = 31; jj >= 0; --jj) {
                        if (jj >= nt) continue;
                        const float u = lane <= jj ? at(jj) : 1.f;
                        if (lane == jj) t = t / u;
                        const float yj = __shfl_sync(0xffffffffu, t, jj);
                        if (lane < jj) t -= u * yj;
                    }
                }
                if (act) y[r0 + lane] = t;
                __syncwarp();
            }
        }
        for (int i = lane; i < m; i += 32) z[(size_t)blk * m + i] = (double)y[i];
        __syncwarp();
    }
}
__global__ void __launch_bounds__(SOLVE_THREADS, 5)
k_lu_solve_half(const __half *__restrict__ pool, const float *__restrict__ row_scale, const int *__restrict__ perm,
                int m, int count, const double *__restrict__ rhs, double *__restrict__ z) {
    lu_solve_half_body(blockIdx.x, gridDim.x, pool, row_scale, perm, m, count, rhs, z);
}

// Transposed block solve z = A^{-T} b with the same slab-layout factors (A = P^T L U, so
// A^{-T} b = P^T L^{-T} U^{-T} b): a forward solve with U^T (lower, with U's diagonal), a
// backward solve with L^T (unit upper), then the scatter z[perm[i]] = x[i].  Slab s holds rows
// 32s.. of U and L; once a slab's unknowns are final, its rows are applied to the remaining
// unknowns with each lane owning one 16-byte column group (no CTA barriers, one warp per block).
template <typename T>
__global__ void __launch_bounds__(SOLVE_THREADS)
k_lu_solve_t(const T *__restrict__ pool, const int *__restrict__ perm, size_t stride, int m, int count,
             const double *__restrict__ rhs, double *__restrict__ z) {
    using SV = SlabVec<T>;
    using V = typename SV::V;
    constexpr int W = SV::W;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    T *y = reinterpret_cast<T *>(smraw) + (size_t)wib * m;
    const int warps = gridDim.x * (SOLVE_THREADS / 32);
    const int slabs = (m + 31) / 32;
    for (int blk = blockIdx.x * (SOLVE_THREADS / 32) + wib; blk < count; blk += warps) {
        const T *A = pool + (size_t)blk * stride;
        const int *pm = perm + (size_t)blk * m;
        const double *b = rhs + (size_t)blk * m;
        for (int i = lane; i < m; i += 32) y[i] = (T)b[i];
        __syncwarp();
        // U^T y = b, forward by slabs
        for (int s = 0; s < slabs; ++s) {
            const int r0 = 32 * s, nt = min(32, m - r0), hi = r0 + nt;
            const T *S = A + (size_t)r0 * m;
            T t = lane < nt ? y[r0 + lane] : T(0);
            for (int jj = 0; jj < nt; ++jj) {
                const T d = lane == jj ? S[slab_at<T>(nt, jj, r0 + jj)] : T(1);
                if (lane == jj) t = t / d;
                const T yj = __shfl_sync(0xffffffffu, t, jj);
                // U^T[r0+lane][r0+jj] = U[r0+jj][r0+lane], nonzero for lane > jj
                if (lane > jj && lane < nt) t -= S[slab_at<T>(nt, jj, r0 + lane)] * yj;
            }
            if (lane < nt) y[r0 + lane] = t;
            __syncwarp();
            for (int g = hi / W + lane; g < m / W; g += 32) {
                T acc[W];
#pragma unroll
                for (int e = 0; e < W; ++e) acc[e] = 0;
                for (int i = 0; i < nt; ++i) {
                    const V v = reinterpret_cast<const V *>(S)[(size_t)g * nt + i];
                    const T yi = y[r0 + i];
                    const T *vv = reinterpret_cast<const T *>(&v);
#pragma unroll
                    for (int e = 0; e < W; ++e) acc[e] += vv[e] * yi;
                }
#pragma unroll
                for (int e = 0; e < W; ++e) y[g * W + e] -= acc[e];
            }
            __syncwarp();
        }
        // L^T x = y (unit upper), backward by slabs
        for (int s = slabs - 1; s >= 0; --s) {
            const int r0 = 32 * s, nt = min(32, m - r0);
            const T *S = A + (size_t)r0 * m;
            T t = lane < nt ? y[r0 + lane] : T(0);
            for (int jj = nt - 1; jj >= 0; --jj) {
                const T yj = __shfl_sync(0xffffffffu, t, jj);
                // L^T[r0+lane][r0+jj] = L[r0+jj][r0+lane], nonzero for lane < jj
                if (lane < jj) t -= S[slab_at<T>(nt, jj, r0 + lane)] * yj;
            }
            if (lane < nt) y[r0 + lane] = t;
            __syncwarp();
            for (int g = lane; g < r0 / W; g += 32) {
                T acc[W];
#pragma unroll
                for (int e = 0; e < W; ++e) acc[e] = 0;
                for (int i = 0; i < nt; ++i) {
                    const V v = reinterpret_cast<const V *>(S)[(size_t)g * nt + i];
                    const T yi = y[r0 + i];
                    const T *vv = reinterpret_cast<const T *>(&v);
#pragma unroll
                    for (int e = 0; e < W; ++e) acc[e] += vv[e] * yi;
                }
#pragma unroll
                for (int e = 0; e < W; ++e) y[g * W + e] -= acc[e];
            }
            __syncwarp();
        }
        for (int i = lane; i < m; i += 32) z[(size_t)blk * m + pm[i]] = (double)y[i];
        __syncwarp();
    }
}

// y = (float) x, elementwise (grid-stride).
__global__ void k_round(const double *__restrict__ x, float *__restrict__ y, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = (float)x[i];
}

// Copy of the factored m x m part of each augmented matrix (row length ld) into the slab
// layout of k_lu_solve (a pool of m x m blocks in TD): one warp per 32-row slab, 16-byte stores.
// Position i's factor row is source row i, or, with perm, source row perm[i] (the left-looking
// LU leaves its factors in original-row order).
template <typename TS, typename TD>
__global__ void k_slab_pack(const TS *__restrict__ src, size_t stride, int m, int ld, int count, TD *__restrict__ dst,
                            const int *__restrict__ perm = nullptr) {
    constexpr int W = SlabVec<TD>::W;
    const int slabs = (m + 31) / 32, lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= (long long)count * slabs) return;
    const int blk = (int)(warp / slabs), s = (int)(warp % slabs), r0 = 32 * s, nt = min(32, m - r0);
    if (lane >= nt) return;
    const int row = perm ? perm[(size_t)blk * m + r0 + lane] : r0 + lane;
    const TS *ar = src + (size_t)blk * stride + (size_t)row * ld;
    TD *out = dst + (size_t)blk * m * m + (size_t)r0 * m;
    for (int g = 0; g < m / W; ++g) {
        typename SlabVec<TD>::V v;
        TD *e = reinterpret_cast<TD *>(&v);
#pragma unroll
        for (int w = 0; w < W; ++w) e[w] = (TD)ar[g * W + w];
        *reinterpret_cast<typename SlabVec<TD>::V *>(out + (size_t)g * nt * W + lane * W) = v;
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

// FP64 multi-RHS back substitution on the tensor pipe: the same blocking as k_backsolve (32-row
// blocks from the bottom, 64 right-hand-side columns at a time), with the update
// X[r0 rows] -= U[r0 rows, l >= hi] X[l rows] done by DMMA: warp w owns the 8 columns
// 8w..8w+7 of the column block and all 32 rows (4 tiles), k-chunks of 32 are staged in shared
// memory with pitches 36 and 68 (4 mod 16) so the fragment loads are conflict-free.
constexpr int BS_RT = 32, BS_CT = 64, BS_KC = 32, BS_UP = 36, BS_XP = 68;
constexpr size_t backsolve_smem_bytes() {
    return sizeof(double) * ((size_t)BS_RT * BS_UP + (size_t)BS_KC * BS_XP + (size_t)BS_RT * (BS_CT + 1) +
                             (size_t)BS_RT * (BS_RT + 1));
}
__global__ void __launch_bounds__(LU_THREADS)
k_backsolve_dmma(double *__restrict__ pool, size_t stride, int m, int ld, int count) {
    extern __shared__ __align__(16) unsigned char smraw[];
    double *Us = reinterpret_cast<double *>(smraw);        // [BS_RT][BS_UP]
    double *Xk = Us + BS_RT * BS_UP;                        // [BS_KC][BS_XP]
    double *Xs = Xk + BS_KC * BS_XP;                        // [BS_RT][BS_CT + 1]
    double *Ud = Xs + BS_RT * (BS_CT + 1);                  // [BS_RT][BS_RT + 1]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, lr = lane >> 2, lc = lane & 3;
    const int nrhs = ld - m;
    for (int blk = blockIdx.x; blk < count; blk += gridDim.x) {
        double *A = pool + (size_t)blk * stride;
        for (int cb = 0; cb < nrhs; cb += BS_CT) {
            const int ct = min(BS_CT, nrhs - cb);
            const int last = ((m - 1) / BS_RT) * BS_RT;
            for (int r0 = last; r0 >= 0; r0 -= BS_RT) {
                const int nt = min(BS_RT, m - r0), hi = r0 + nt;
                double c[4][2];
#pragma unroll
                for (int mt = 0; mt < 4; ++mt)
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const int r = mt * 8 + lr, col = warp * 8 + 2 * lc + e;
                        c[mt][e] = (r < nt && col < ct) ? A[(size_t)(r0 + r) * ld + m + cb + col] : 0.;
                    }
                for (int l0 = hi; l0 < m; l0 += BS_KC) {
                    const int kc = min(BS_KC, m - l0);
                    for (int idx = tid; idx < BS_RT * BS_KC; idx += LU_THREADS) {
                        const int r = idx / BS_KC, l = idx % BS_KC;
                        Us[r * BS_UP + l] = (r < nt && l < kc) ? A[(size_t)(r0 + r) * ld + l0 + l] : 0.;
                    }
                    for (int idx = tid; idx < BS_KC * BS_CT; idx += LU_THREADS) {
                        const int l = idx / BS_CT, col = idx % BS_CT;
                        Xk[l * BS_XP + col] = (l < kc && col < ct) ? A[(size_t)(l0 + l) * ld + m + cb + col] : 0.;
                    }
                    __syncthreads();
                    for (int kk = 0; kk < kc; kk += 4) {
                        const double b = Xk[(kk + lc) * BS_XP + warp * 8 + lr];
#pragma unroll
                        for (int mt = 0; mt < 4; ++mt) dmma8x8x4(c[mt], -Us[(mt * 8 + lr) * BS_UP + kk + lc], b);
                    }
                    __syncthreads();
                }
#pragma unroll
                for (int mt = 0; mt < 4; ++mt)
#pragma unroll
                    for (int e = 0; e < 2; ++e) Xs[(mt * 8 + lr) * (BS_CT + 1) + warp * 8 + 2 * lc + e] = c[mt][e];
                for (int idx = tid; idx < BS_RT * BS_RT; idx += LU_THREADS) {
                    const int r = idx / BS_RT, col = idx % BS_RT;
                    Ud[r * (BS_RT + 1) + col] = (r < nt && col < nt) ? A[(size_t)(r0 + r) * ld + r0 + col] : 0.;
                }
                __syncthreads();
                if (tid < ct)
                    for (int i = nt - 1; i >= 0; --i) {
                        double val = Xs[i * (BS_CT + 1) + tid];
                        for (int l = i + 1; l < nt; ++l) val -= Ud[i * (BS_RT + 1) + l] * Xs[l * (BS_CT + 1) + tid];
                        Xs[i * (BS_CT + 1) + tid] = val / Ud[i * (BS_RT + 1) + i];
                    }
                __syncthreads();
                for (int idx = tid; idx < nt * ct; idx += LU_THREADS) {
                    const int r = idx / ct, col = idx % ct;
                    A[(size_t)(r0 + r) * ld + m + cb + col] = Xs[r * (BS_CT + 1) + col];
                }
                __syncthreads();
            }
        }
    }
}

}  // namespace dgh
