// Block ILU(0) of the 1D solver (dg_hdg_1d --precond block-ilu0): BlockPreconditioner on
// BlockGraph::periodic(cells) in the natural ordering (common/src/linalg/block_ilu.cpp:15-84,
// block_graph.cpp:30-35).  The factorisation and the two triangular sweeps are sequential over
// block rows (row i needs row i-1), so each runs as one CTA that walks the rows in the
// reference's order and spreads the work inside a row (block rows, block products, the dense
// pivoted LU of the diagonal block) over its threads.  The pattern and the symbolic update
// schedule (block_ilu.cpp:24-45) are built once on the host.  Blocks are row-major m x m in
// pattern-slot order; the LU of a diagonal block replaces it in place with its row
// permutation in perm[row * m ..].
#pragma once
#include "dgh_kernels_1d.cuh"

namespace dgh {

constexpr int ILU_THREADS = 256;

// Every pattern block (dg_operator.cpp:50-78): the volume block and the mass diagonal on the
// diagonal, and the face terms of the two faces of block row R that land in column C (with
// one or two cells, several land in the same block).
template <int N, typename TF>
__global__ void k1_ilu_dg_blocks(TF *__restrict__ vals, const int *__restrict__ slot_row, const int *__restrict__ col_idx,
                                 int nnz, const double *__restrict__ jq, const double *__restrict__ fj, Basis1Q b,
                                 Grid1 g, double inv_step) {
    constexpr int M = NV1 * N;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)nnz * M * M) return;
    const int slot = (int)(idx / (M * M)), e = (int)(idx % (M * M)), row = e / M, col = e % M;
    const int R = slot_row[slot], C = col_idx[slot];
    const int v = row / N, i = row % N, w = col / N, j = col % N;
    double val = 0;
    if (R == C) {
        val = vol_entry1<N>(b, jq, R, v, i, w, j);
        if (row == col) val += .5 * g.h * b.w[i] * inv_step;
    }
    const int prev = R == 0 ? g.cells - 1 : R - 1, next = R + 1 == g.cells ? 0 : R + 1;
    // side 0: face prev (test: left values, sign -1); trace side 0 is the left cell prev, 1 is R
    if (C == prev) val += -b.eL[i] * b.eR[j] * fj[(size_t)prev * 18 + v * 3 + w];
    if (C == R) val += -b.eL[i] * b.eL[j] * fj[(size_t)prev * 18 + 9 + v * 3 + w];
    // side 1: face R (test: right values, sign +1); trace side 0 is R, 1 is next
    if (C == R) val += b.eR[i] * b.eR[j] * fj[(size_t)R * 18 + v * 3 + w];
    if (C == next) val += b.eR[i] * b.eL[j] * fj[(size_t)R * 18 + 9 + v * 3 + w];
    vals[idx] = (TF)val;
}

// Every pattern block of the condensed trace operator (hybrid.cpp:104-117): -(a + b) I on the
// diagonal plus, for the two cells beside face F, their Schur blocks whose column face is C.
template <typename TF>
__global__ void k1_ilu_face_blocks(TF *__restrict__ vals, const int *__restrict__ slot_row,
                                   const int *__restrict__ col_idx, int nnz, const double *__restrict__ S,
                                   const double *__restrict__ speeds, Grid1 g) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nnz * 9) return;
    const int slot = idx / 9, v = (idx % 9) / 3, w = idx % 3;
    const int F = slot_row[slot], C = col_idx[slot];
    double val = F == C && v == w ? -(speeds[2 * F] + speeds[2 * F + 1]) : 0.;
    for (int adjacent = 0; adjacent < 2; ++adjacent) {
        const int cell = (F + adjacent) % g.cells, row_side = adjacent == 0 ? 1 : 0;
        for (int col_side = 0; col_side < 2; ++col_side) {
            const int face = col_side == 0 ? (cell == 0 ? g.cells - 1 : cell - 1) : cell;
            if (face == C) val += S[(size_t)cell * T1 * T1 + (row_side * NV1 + v) * T1 + col_side * NV1 + w];
        }
    }
    vals[idx] = (TF)val;
}

// Pivoted LU (dense_lu.hpp:10-16) of the m x m (m <= 32) block A in place by warp 0, lane r
// owning row r; perm[r] = original row at position r.  Returns the status bit to raise (0 if
// the block and its factors are valid) to every thread of the CTA.
template <typename TF>
__device__ int ilu_block_lu(TF *A, int *perm, int m, int *flag) {
    const int tid = threadIdx.x, lane = tid & 31;
    __syncthreads();  // every thread has read the flag of the previous block
    if (tid == 0) *flag = 0;
    __syncthreads();
    bool bad_in = false;
    for (int k = tid; k < m * m; k += blockDim.x) bad_in = bad_in || !isfinite((double)A[k]);
    if (bad_in) atomicOr(flag, ST_LU_INPUT);
    __syncthreads();
    if (*flag) return *flag;
    if (tid < 32) {
        int orig = lane;
        for (int j = 0; j < m; ++j) {
            TF best = TF(-1);
            int bi = 0x7fffffff;
            if (lane >= j && lane < m) {
                const TF a = A[lane * m + j];
                if (a == a) {
                    best = a < TF(0) ? -a : a;
                    bi = lane;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const TF ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
            }
            const int p = __shfl_sync(0xffffffffu, bi == 0x7fffffff ? j : bi, 0);
            if (p != j) {
                for (int c = lane; c < m; c += 32) {
                    const TF t = A[j * m + c];
                    A[j * m + c] = A[p * m + c];
                    A[p * m + c] = t;
                }
                const int oj = __shfl_sync(0xffffffffu, orig, j), op = __shfl_sync(0xffffffffu, orig, p);
                if (lane == j) orig = op;
                if (lane == p) orig = oj;
            }
            __syncwarp();
            const TF pivot = A[j * m + j];
            if (lane > j && lane < m) {
                TF *Ar = A + lane * m;
                const TF l = pivot != TF(0) ? Ar[j] / pivot : Ar[j];
                Ar[j] = l;
                const TF *Aj = A + j * m;
                for (int c = j + 1; c < m; ++c) Ar[c] -= l * Aj[c];
            }
            __syncwarp();
        }
        bool bad = false;
        for (int k = lane; k < m * m; k += 32) bad = bad || !isfinite((double)A[k]);
        if (lane < m) {
            bad = bad || !(fabs((double)A[lane * m + lane]) > 2.2250738585072014e-308);
            perm[lane] = orig;
        }
        if (__any_sync(0xffffffffu, bad) && lane == 0) *flag = ST_SINGULAR_HDG;
    }
    __syncthreads();
    return *flag;
}

// block_ilu.cpp:48-61: for each row i, for each block left of the diagonal, X <- X D_j^{-1}
// (dense_lu.hpp:42-49: U^T, then L^T, then P^T, row by row) and the scheduled updates
// C -= X U (dense_lu.hpp:53-57, k ascending per entry), then the LU of the diagonal block.
// One CTA; stops at the first failing block and raises its status bit.
template <typename TF>
__global__ void __launch_bounds__(ILU_THREADS)
k1_ilu_factor(TF *__restrict__ vals, int *__restrict__ perm, const int *__restrict__ row_ptr,
              const int *__restrict__ col_idx, const int *__restrict__ diag, const int *__restrict__ upd_off,
              const int *__restrict__ upd_target, const int *__restrict__ upd_upper, int rows, int m,
              int *status) {
    __shared__ int flag;
    __shared__ double s[32 * 33];  // one row of X per thread (m <= 32)
    const size_t m2 = (size_t)m * m;
    const int tid = threadIdx.x;
    for (int i = 0; i < rows; ++i) {
        for (int p = row_ptr[i]; p < diag[i]; ++p) {
            const int j = col_idx[p];
            TF *X = vals + (size_t)p * m2;
            const TF *D = vals + (size_t)diag[j] * m2;
            const int *pj = perm + (size_t)j * m;
            if (tid < m) {  // row tid of X
                double *t = s + tid * 33;
                for (int k = 0; k < m; ++k) t[k] = (double)X[tid * m + k];
                for (int a = 0; a < m; ++a) {  // U^T t' = t
                    double v = t[a];
                    for (int k = 0; k < a; ++k) v -= (double)D[k * m + a] * t[k];
                    t[a] = v / (double)D[a * m + a];
                }
                for (int a = m - 1; a >= 0; --a) {  // L^T t'' = t'
                    double v = t[a];
                    for (int k = a + 1; k < m; ++k) v -= (double)D[k * m + a] * t[k];
                    t[a] = v;
                }
                for (int a = 0; a < m; ++a) X[tid * m + pj[a]] = (TF)t[a];
            }
            __syncthreads();
            for (int u = upd_off[p]; u < upd_off[p + 1]; ++u) {
                TF *Cb = vals + (size_t)upd_target[u] * m2;
                const TF *Rb = vals + (size_t)upd_upper[u] * m2;
                for (int e = tid; e < m * m; e += blockDim.x) {
                    const int q = e / m, c = e % m;
                    TF acc = Cb[e];
                    for (int k = 0; k < m; ++k) acc -= Rb[k * m + c] * X[q * m + k];
                    Cb[e] = acc;
                }
                __syncthreads();
            }
        }
        const int f = ilu_block_lu(vals + (size_t)diag[i] * m2, perm + (size_t)i * m, m, &flag);
        if (f) {
            if (tid == 0) atomicOr(status, f);
            return;
        }
    }
}

// block_ilu.cpp:62-84 in the natural order: z = x; forward z_i -= L_ip z_col (blocks left of the
// diagonal); backward z_i -= U_ip z_col (blocks right of it), then z_i = D_i^{-1} z_i (P, unit
// L, U).  One CTA; the block products accumulate in FP64 whatever the storage type.
template <typename TF>
__global__ void __launch_bounds__(ILU_THREADS)
k1_ilu_apply(const TF *__restrict__ vals, const int *__restrict__ perm, const int *__restrict__ row_ptr,
             const int *__restrict__ col_idx, const int *__restrict__ diag, int rows, int m,
             const double *__restrict__ x, double *__restrict__ z) {
    const size_t m2 = (size_t)m * m;
    const int tid = threadIdx.x, lane = tid & 31;
    for (long long e = tid; e < (long long)rows * m; e += blockDim.x) z[e] = x[e];
    __syncthreads();
    for (int i = 0; i < rows; ++i) {
        for (int p = row_ptr[i]; p < diag[i]; ++p) {
            const TF *B = vals + (size_t)p * m2;
            const double *zc = z + (size_t)col_idx[p] * m;
            double s = 0;
            if (tid < m)
                for (int k = 0; k < m; ++k) s += (double)B[tid * m + k] * zc[k];
            __syncthreads();
            if (tid < m) z[(size_t)i * m + tid] -= s;
            __syncthreads();
        }
    }
    for (int i = rows - 1; i >= 0; --i) {
        for (int p = diag[i] + 1; p < row_ptr[i + 1]; ++p) {
            const TF *B = vals + (size_t)p * m2;
            const double *zc = z + (size_t)col_idx[p] * m;
            double s = 0;
            if (tid < m)
                for (int k = 0; k < m; ++k) s += (double)B[tid * m + k] * zc[k];
            __syncthreads();
            if (tid < m) z[(size_t)i * m + tid] -= s;
            __syncthreads();
        }
        if (tid < 32) {
            const TF *D = vals + (size_t)diag[i] * m2;
            const int *pi = perm + (size_t)i * m;
            double *zi = z + (size_t)i * m;
            const bool act = lane < m;
            double y = act ? zi[pi[lane]] : 0.;
            for (int j = 0; j < m; ++j) {
                const double yj = __shfl_sync(0xffffffffu, y, j);
                if (act && lane > j) y -= (double)D[lane * m + j] * yj;
            }
            for (int j = m - 1; j >= 0; --j) {
                if (lane == j) y = y / (double)D[j * m + j];
                const double yj = __shfl_sync(0xffffffffu, y, j);
                if (act && lane < j) y -= (double)D[lane * m + j] * yj;
            }
            __syncwarp();
            if (act) zi[lane] = y;
        }
        __syncthreads();
    }
}

}  // namespace dgh
