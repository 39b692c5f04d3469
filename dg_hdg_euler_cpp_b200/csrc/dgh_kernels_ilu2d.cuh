// 2D block ILU(0) of the DG Jacobian on the periodic cartesian block graph in the natural
// ordering (common/src/linalg/block_ilu.cpp:15-84 restated for the 2D operator; the reference's
// 2D front end offers block Jacobi only).  Kernels: the face coupling blocks of DGOperator::block
// (dg_operator.cpp:22-48, col != row), the level-scheduled forward and backward sweeps of the
// application, and the gathers of the factorisation.  The batched block products of the
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

// Block row product acc[r] = sum_j blk[r][j] x[j] for the CTA's m rows: warp per row, lanes over
// the row's contiguous entries, FP64 accumulation.
template <typename TF>
__device__ inline double row_dot(const TF *__restrict__ row, const double *__restrict__ x, int m) {
    const int lane = threadIdx.x & 31;
    double acc = 0;
    for (int j = lane; j < m; j += 32) acc += (double)row[j] * x[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    return acc;
}

// Forward sweep of one level (block_ilu.cpp:70-74): for each listed row i,
// work_i -= sum over its lower slots p of L_p work_col(p).  One CTA per row.
template <typename TF>
__global__ void __launch_bounds__(256)
k_ilu2_forward(const int *__restrict__ rows, int count, const int *__restrict__ nlower, const int *__restrict__ ncol,
               const TF *__restrict__ offd, double *__restrict__ work, int m) {
    extern __shared__ double xs[];  // the lower neighbours' work segments, 4 m at most
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int k = blockIdx.x; k < count; k += gridDim.x) {
        const int i = rows[k], nl = nlower[i];
        __syncthreads();
        for (int p = 0; p < nl; ++p)
            for (int j = threadIdx.x; j < m; j += blockDim.x) xs[p * m + j] = work[(size_t)ncol[4 * i + p] * m + j];
        __syncthreads();
        for (int r = warp; r < m; r += blockDim.x / 32) {
            double s = 0;
            for (int p = 0; p < nl; ++p) s += row_dot(offd + ((size_t)(4 * i + p) * m + r) * m, xs + p * m, m);
            if (lane == 0) work[(size_t)i * m + r] -= s;
        }
    }
}

// Backward sweep of one level (block_ilu.cpp:75-80): for each listed row i,
// z_i = A_ii^{-1} (work_i - sum over its upper slots p of U_p z_col(p)), the inverse stored over
// the diagonal block.  One CTA per row.
template <typename TF>
__global__ void __launch_bounds__(256)
k_ilu2_backward(const int *__restrict__ rows, int count, const int *__restrict__ nlower, const int *__restrict__ ncol,
                const TF *__restrict__ offd, const TF *__restrict__ diag, const double *__restrict__ work,
                double *__restrict__ z, int m) {
    extern __shared__ double xs[];  // the upper neighbours' z segments (4 m at most), then t (m)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *t = xs + 4 * m;
    for (int k = blockIdx.x; k < count; k += gridDim.x) {
        const int i = rows[k], nl = nlower[i];
        __syncthreads();
        for (int p = nl; p < 4; ++p)
            for (int j = threadIdx.x; j < m; j += blockDim.x) xs[p * m + j] = z[(size_t)ncol[4 * i + p] * m + j];
        __syncthreads();
        for (int r = warp; r < m; r += blockDim.x / 32) {
            double s = 0;
            for (int p = nl; p < 4; ++p) s += row_dot(offd + ((size_t)(4 * i + p) * m + r) * m, xs + p * m, m);
            if (lane == 0) t[r] = work[(size_t)i * m + r] - s;
        }
        __syncthreads();
        for (int r = warp; r < m; r += blockDim.x / 32) {
            const double s = row_dot(diag + ((size_t)i * m + r) * m, t, m);
            if (lane == 0) z[(size_t)i * m + r] = s;
        }
    }
}

}  // namespace dgh
