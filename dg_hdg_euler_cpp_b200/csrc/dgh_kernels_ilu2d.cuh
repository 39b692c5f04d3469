// 2D block ILU(0) of the DG Jacobian on the periodic cartesian block graph in the natural
// ordering (common/src/linalg/block_ilu.cpp:15-84 restated for the 2D operator; the reference's
// 2D front end offers block Jacobi only).  Kernels: the face coupling blocks of DGOperator::block
// (dg_operator.cpp:22-48, col != row), the level-scheduled forward and backward sweeps of the
// application, and the block copies and inverse staging of the factorisation.  The batched block products of the
// factorisation are plain GEMMs (cuBLAS), and the diagonal inverses come from k_lu_left.
#pragma once
#include "dgh_kernels_dg.cuh"

namespace dgh {

// Coupling block of cell `cell` to its neighbour across `side` (dg_operator.cpp:22-48 with
// col = neighbor(row, side)), row-major m x m, m = 4 N^2: the HLL derivative with respect to the
// neighbour's face state (face_jacobian.cpp:69-73), restricted from the neighbour's face line and
// lifted on this cell's, with the lift sign of this cell's side.  One CTA per (cell, side) pair
// of the list; dst[k] is the block of pair k.
template <int N, typename TF>
__global__ void __launch_bounds__(256)
k_dg_coupling(TF *const *__restrict__ dst, const int *__restrict__ pairs, int count, const double *__restrict__ fcache,
              const double *__restrict__ speeds, Basis1D b, Grid g) {
    constexpr int P = N * N, M = NVAR * P;
    __shared__ double G[N * 16];
    __shared__ Basis1D sb;
    stage_basis<N>(b, sb);
    for (int k = blockIdx.x; k < count; k += gridDim.x) {
        const int cell = pairs[2 * k], side = pairs[2 * k + 1];
        const int face = face_of(g, cell, side), axis = side / 2;
        const bool left_col = side % 2 == 0;  // the neighbour is the face's left state on sides 0 and 2
        const double sign = side % 2 ? 1. : -1.;
        __syncthreads();
        for (int q = threadIdx.x; q < N; q += blockDim.x) {
            const double *c = fcache + ((size_t)face * N + q) * 8;
            const double sa = speeds[2 * (face * N + q)], sbb = speeds[2 * (face * N + q) + 1];
            const double pen = face_weight(g, sb, face, q) * sa * sbb / (sa + sbb);
            double a[16];
            if (left_col) cached_jacobian(g.gamma, c[0], c[1], c[2], axis, a);
            else cached_jacobian(g.gamma, c[3], c[4], c[5], axis, a);
            const double blend = left_col ? c[6] : c[7];
#pragma unroll
            for (int v = 0; v < 4; ++v)
#pragma unroll
                for (int w = 0; w < 4; ++w)
                    G[q * 16 + v * 4 + w] = sign * (a[v * 4 + w] * blend + (v == w ? (left_col ? pen : -pen) : 0.));
        }
        __syncthreads();
        const double *test = side % 2 ? sb.eR : sb.eL, *trial = left_col ? sb.eR : sb.eL;
        TF *out = dst[k];
        for (int idx = threadIdx.x; idx < M * M; idx += blockDim.x) {
            const int r = idx / M, c = idx % M;
            const int v = r / P, rn = r % P, ix = rn % N, iy = rn / N;
            const int w = c / P, cn = c % P, jx = cn % N, jy = cn / N;
            double val = 0;
            if (side < 2) {
                if (iy == jy) val = G[iy * 16 + v * 4 + w] * test[ix] * trial[jx];
            } else if (ix == jx) {
                val = G[ix * 16 + v * 4 + w] * test[iy] * trial[jy];
            }
            out[idx] = (TF)val;
        }
    }
}

// Copies count m x m blocks: dst[k] = src[k] (the factorisation's products land in scratch first).
template <typename TF>
__global__ void k_copy_blocks(TF *const *__restrict__ dst, const TF *const *__restrict__ src, int count, int mm) {
    for (int k = blockIdx.x; k < count; k += gridDim.x) {
        const TF *s = src[k];
        TF *d = dst[k];
        for (int i = threadIdx.x; i < mm; i += blockDim.x) d[i] = s[i];
    }
}

// [A_ii | I | 0] in FP64 (row length 2m + 1) from the stored diagonal blocks of the listed rows,
// for k_lu_left's augmented solve: X = A_ii^{-1}.
template <typename TF>
__global__ void k_ilu_stage_inverse(double *__restrict__ aug, const TF *__restrict__ diag, const int *__restrict__ rows,
                                    int count, int m) {
    const int ld = 2 * m + 1;
    for (int k = blockIdx.x; k < count; k += gridDim.x) {
        const TF *a = diag + (size_t)rows[k] * m * m;
        double *o = aug + (size_t)k * m * ld;
        for (int idx = threadIdx.x; idx < m * ld; idx += blockDim.x) {
            const int r = idx / ld, c = idx % ld;
            o[idx] = c < m ? (double)a[(size_t)r * m + c] : (c - m == r ? 1. : 0.);
        }
    }
}

// Stores the inverses (row-major, FP64) of the listed rows over their diagonal blocks, rounded to TF.
template <typename TF>
__global__ void k_ilu_store_inverse(TF *__restrict__ diag, const double *__restrict__ inv, const int *__restrict__ rows,
                                    int count, int m) {
    for (int k = blockIdx.x; k < count; k += gridDim.x) {
        TF *d = diag + (size_t)rows[k] * m * m;
        const double *s = inv + (size_t)k * m * m;
        for (int i = threadIdx.x; i < m * m; i += blockDim.x) d[i] = (TF)s[i];
    }
}

// The sweeps of one level, split over CTAs: CTA (k, chunk) computes output rows
// [ILU_ROWS chunk, ILU_ROWS (chunk + 1)) of the level's k-th block row, one warp per output row
// with 16-byte loads of the block rows (all blocks of the output row in flight together) and the
// right-hand-side segments staged in shared memory.
//   MODE 0 (forward, block_ilu.cpp:70-74):   work_i -= sum_{lower p} L_p work_col(p)
//   MODE 1 (backward, the upper products):   t_i = work_i - sum_{upper p} U_p z_col(p)
//   MODE 2 (backward, the diagonal):         z_i = A_ii^{-1} t_i
constexpr int ILU_ROWS = 32;
template <typename TF> struct IluVec;
template <> struct IluVec<double> { using V = double2; static constexpr int W = 2; };
template <> struct IluVec<float> { using V = float4; static constexpr int W = 4; };

template <typename TF, int MODE>
__global__ void __launch_bounds__(256)
k_ilu2_rows(const int *__restrict__ rows, int count, int chunks, const int *__restrict__ nlower,
            const int *__restrict__ ncol, const TF *__restrict__ offd, const TF *__restrict__ diag,
            double *work, double *__restrict__ t, double *__restrict__ z, int m) {
    using V = typename IluVec<TF>::V;
    constexpr int W = IluVec<TF>::W;
    extern __shared__ __align__(16) double xs[];  // up to 4 segments of m
    const int k = blockIdx.x / chunks, chunk = blockIdx.x % chunks;
    if (k >= count) return;
    const int i = rows[k], nl = nlower[i];
    const int p0 = MODE == 0 ? 0 : MODE == 1 ? nl : 0, p1 = MODE == 0 ? nl : MODE == 1 ? 4 : 1;
    for (int p = p0; p < p1; ++p) {
        const double *src = MODE == 0 ? work + (size_t)ncol[4 * i + p] * m
                            : MODE == 1 ? z + (size_t)ncol[4 * i + p] * m : t + (size_t)i * m;
        for (int j = threadIdx.x; j < m; j += blockDim.x) xs[(p - p0) * m + j] = src[j];
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, G = m / W;
    for (int r = chunk * ILU_ROWS + warp; r < min(m, (chunk + 1) * ILU_ROWS); r += blockDim.x / 32) {
        double acc = 0;
        for (int p = p0; p < p1; ++p) {
            const TF *blk = MODE == 2 ? diag + (size_t)i * m * m : offd + (size_t)(4 * i + p) * m * m;
            const V *row = reinterpret_cast<const V *>(blk + (size_t)r * m);
            const double *x = xs + (p - p0) * m;
            for (int g = lane; g < G; g += 32) {
                const V a = row[g];
                const TF *e = reinterpret_cast<const TF *>(&a);
#pragma unroll
                for (int w = 0; w < W; ++w) acc += (double)e[w] * x[g * W + w];
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) {
            const size_t at = (size_t)i * m + r;
            if (MODE == 0) work[at] -= acc;
            else if (MODE == 1) t[at] = work[at] - acc;
            else z[at] = acc;
        }
    }
}

}  // namespace dgh
