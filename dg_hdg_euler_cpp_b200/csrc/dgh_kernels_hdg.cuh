// HDG static condensation (hybrid.cpp): per-cell augmented matrix [A | B | r], whose LU with
// forward elimination and back substitution yields X = A^{-1}B and y = A^{-1}r; the local
// Schur block S_K = -C X and C y (face_jacobian.cpp:88-110); face-block Jacobi blocks
// (hybrid.cpp:83-96); the face-owned Schur apply (hybrid.cpp:73-82); recovery
// du = -X dlambda - y (hybrid.cpp:97-105) and the recovered DG residual (hybrid.cpp:106-121).
#pragma once
#include "dgh_kernels_dg.cuh"

namespace dgh {

// Augmented rows [m][ld], ld = m + t + 1, t = 16 N, for cells first..first+count-1.
template <int N, typename TF>
__global__ void __launch_bounds__(256)
k_hdg_assemble(TF *__restrict__ aug, const double *__restrict__ vol, const double *__restrict__ fcache,
               const double *__restrict__ speeds, const double *__restrict__ rvol, Basis1D b, Grid g,
               double inv_step, int first, int count, int volterm = 1) {
    constexpr int P = N * N, M = NVAR * P, FW = NVAR * N, T = NFACES * FW, LD = M + T + 1;
    __shared__ double jx[P * 16], jy[P * 16], fj[NFACES * N * 16], stab[NFACES * N];
    __shared__ Basis1D sb;
    stage_basis<N>(b, sb);
    for (int blk = blockIdx.x; blk < count; blk += gridDim.x) {
        const int cell = first + blk;
        __syncthreads();
        cell_tables<N, true>(cell, vol, fcache, speeds, sb, g, jx, jy, fj);
        for (int k = threadIdx.x; k < NFACES * N; k += blockDim.x) {
            const int side = k / N, q = k % N, face = face_of(g, cell, side);
            const double tau = speeds[2 * (face * N + q) + (side % 2 ? 0 : 1)];
            stab[k] = face_weight(g, sb, face, q) * tau;
        }
        __syncthreads();
        TF *A = aug + (size_t)blk * M * LD;
        for (int idx = threadIdx.x; idx < M * LD; idx += blockDim.x) {
            const int r = idx / LD, c = idx % LD;
            double val;
            if (c < M) {
                val = cell_block_entry<N>(r, c, jx, jy, fj, sb, g, inv_step, volterm != 0);
            } else if (c < M + T) {
                const int k = c - M, side = k / FW, rem = k % FW, vv = rem / N, q = rem % N;
                const int v = r / P, node = r % P, ix = node % N, iy = node / N;
                val = 0;
                if (v == vv) {
                    const double *e = side % 2 ? sb.eR : sb.eL;
                    if (side < 2 && iy == q) val = -stab[side * N + q] * e[ix];
                    if (side >= 2 && ix == q) val = -stab[side * N + q] * e[iy];
                }
            } else {
                val = rvol[(size_t)cell * M + r];
            }
            A[idx] = (TF)val;
        }
    }
}

// From the solved columns [X | y] of every cell: S_K = -(C X) (t x t, row-major, stored as TS)
// and cy = C y.  IN_X: the condensation LU wrote X (m x t row-major) and y straight to their
// persistent arrays; otherwise they are read from the augmented workspace (ld = m + t + 1) and
// copied out (X only where X is not null: the FP32 condensation keeps the LU factors instead).
// Each thread restricts one solved column to one line of face nodes for both faces of an axis
// (the two faces read the same line with the eL and eR weights), so every solved value is read
// twice instead of four times.  col0 = T restricts the work to the y column (cy = C y alone,
// IN_X, for a right-hand side solved against stored factors).
template <int N, typename TF, bool IN_X, typename TS = double>
__global__ void __launch_bounds__(256)
k_hdg_schur(const TF *__restrict__ aug, const double *__restrict__ fcache, const double *__restrict__ speeds,
            TS *__restrict__ S, double *__restrict__ X, double *__restrict__ y, double *__restrict__ cy,
            Basis1D b, Grid g, int first, int count, int col0 = 0) {
    constexpr int P = N * N, M = NVAR * P, FW = NVAR * N, T = NFACES * FW, LD = M + T + 1;
    const int ncol = T + 1 - col0;
    __shared__ double G[NFACES * N * 16];
    for (int blk = blockIdx.x; blk < count; blk += gridDim.x) {
        const int cell = first + blk;
        __syncthreads();
        for (int k = threadIdx.x; k < NFACES * N; k += blockDim.x) {
            const int side = k / N, q = k % N, face = face_of(g, cell, side), axis = side / 2;
            const bool left = side % 2;
            const double *c = fcache + ((size_t)face * N + q) * 8;
            const double sa = speeds[2 * (face * N + q)], sb = speeds[2 * (face * N + q) + 1];
            const double w = face_weight(g, b, face, q), sign = left ? 1. : -1., tau = left ? sa : sb;
            double a[16];
            if (left) cached_jacobian(g.gamma, c[0], c[1], c[2], axis, a);
            else cached_jacobian(g.gamma, c[3], c[4], c[5], axis, a);
#pragma unroll
            for (int v = 0; v < 4; ++v)
#pragma unroll
                for (int ww = 0; ww < 4; ++ww)
                    G[k * 16 + v * 4 + ww] = (sign * a[v * 4 + ww] + (v == ww ? tau : 0.)) * w;
        }
        __syncthreads();
        const TF *A = aug ? aug + (size_t)blk * M * LD : nullptr;
        const double *Xc = X ? X + (size_t)cell * M * T : nullptr, *yc = y + (size_t)cell * M;
        // C applied to every solved column: restrict to the (axis, q) line, then the 4x4 derivative
        for (int idx = threadIdx.x; idx < 2 * N * ncol; idx += blockDim.x) {
            const int col = col0 + idx % ncol, aq = idx / ncol, axis = aq / N, q = aq % N;
            double rl[4], rr[4];
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                double sl = 0, sr = 0;
#pragma unroll
                for (int i = 0; i < N; ++i) {
                    const int r = w * P + face_node(N, 2 * axis, q, i);
                    const double val = IN_X ? (col < T ? Xc[(size_t)r * T + col] : yc[r])
                                            : (double)A[(size_t)r * LD + M + col];
                    sl += b.eL[i] * val;
                    sr += b.eR[i] * val;
                }
                rl[w] = sl;
                rr[w] = sr;
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int side = 2 * axis + h, sq = side * N + q;
                const double *rv = h ? rr : rl;
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    double s = 0;
#pragma unroll
                    for (int w = 0; w < 4; ++w) s += rv[w] * G[sq * 16 + v * 4 + w];
                    const int row = side * FW + v * N + q;
                    if (col < T) S[(size_t)cell * T * T + (size_t)row * T + col] = (TS)(-s);
                    else cy[(size_t)cell * T + row] = s;
                }
            }
        }
        if (!IN_X)
            for (int idx = threadIdx.x; idx < M * (T + 1); idx += blockDim.x) {
                const int r = idx / (T + 1), c = idx % (T + 1);
                const double val = (double)A[(size_t)r * LD + M + c];
                if (c < T) {
                    if (X) X[(size_t)cell * M * T + (size_t)r * T + c] = val;
                } else {
                    y[(size_t)cell * M + r] = val;
                }
            }
    }
}

// Condensed right-hand side: rhs_f = -g_f + sum of the two adjacent cells' C y slots (g = 0
// on the projected trace, hybrid.cpp:28-30).
template <int N>
__global__ void k_hdg_rhs(const double *__restrict__ cy, double *__restrict__ rhs, Grid g) {
    constexpr int FW = NVAR * N, T = NFACES * FW;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 2 * g.cells * FW) return;
    const int face = idx / FW, k = idx % FW, axis = face >= g.cells, first = face - axis * g.cells;
    const int next = neighbor(g, first, 2 * axis + 1);
    rhs[idx] = cy[(size_t)first * T + (2 * axis + 1) * FW + k] + cy[(size_t)next * T + (2 * axis) * FW + k];
}

// Face-block Jacobi blocks D + S_first[rs, rs] + S_next[rs', rs'] written row-major (fw x fw).
template <int N, typename TF, typename TS = double>
__global__ void k_face_blocks(const TS *__restrict__ S, const double *__restrict__ speeds,
                              TF *__restrict__ pool, Basis1D b, Grid g) {
    constexpr int FW = NVAR * N, T = NFACES * FW;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)2 * g.cells * FW * FW) return;
    const int face = idx / (FW * FW), e = idx % (FW * FW), i = e / FW, j = e % FW;
    const int axis = face >= g.cells, first = face - axis * g.cells, next = neighbor(g, first, 2 * axis + 1);
    const int rs = 2 * axis + 1, rn = 2 * axis;
    double val = 0;
    if (i == j) {
        const int q = i % N;
        val = -face_weight(g, b, face, q) * (speeds[2 * (face * N + q)] + speeds[2 * (face * N + q) + 1]);
    }
    val += (double)S[(size_t)first * T * T + (size_t)(rs * FW + i) * T + rs * FW + j];
    val += (double)S[(size_t)next * T * T + (size_t)(rn * FW + i) * T + rn * FW + j];
    pool[idx] = (TF)val;
}

// Face-owned Schur apply: out_f = D_f l_f + S_first[rs rows] l(first) + S_next[rs' rows] l(next).
template <int N>
__global__ void __launch_bounds__(256)
k_hdg_apply(const double *__restrict__ S, const double *__restrict__ speeds, const double *__restrict__ lam,
            double *__restrict__ out, Basis1D b, Grid g);
// The same with FP32 Schur blocks (the FP32 condensation), products and sums in FP64, so the
// operator applied is exactly the stored FP32 S.  The FP32 -> FP64 widening is done on the
// integer pipe: a float's bit pattern shifted right by 3 (sign kept) and its low mantissa bits
// shifted into the low word is the double v * 2^-896, exactly, for every finite v (zero and
// subnormals included); the gathered trace values are stored scaled by 2^896, so each product
// is exact and no conversion instruction is issued per S entry.  (Non-finite S entries would
// not survive this widening; the condensation's factor check rejects non-finite factors.)
__device__ __forceinline__ double widen_scaled(float f) {
    const unsigned b = __float_as_uint(f);
    return __hiloint2double((int)(((b & 0x7fffffffu) >> 3) | (b & 0x80000000u)), (int)(b << 29));
}
// (The Schur-apply bodies take their face explicitly, so the batched kernels of a lockstep
// batch run the same arithmetic per member; every rounding is explicit: fma() and rfma.)
template <int N>
__device__ __forceinline__ void hdg_apply32_body(int face, const float *__restrict__ S, const double *__restrict__ speeds,
                                                 const double *__restrict__ lam, double *__restrict__ out,
                                                 const Basis1D &b, const Grid &g) {
    constexpr int FW = NVAR * N, T = NFACES * FW, T4 = T / 4, PASSES = (T4 + 31) / 32;
    constexpr double kScale = 0x1p896;  // undoes the 2^-896 of widen_scaled
    __shared__ __align__(16) double loc[2][T];
    const int axis = face >= g.cells, first = face - axis * g.cells, next = neighbor(g, first, 2 * axis + 1);
    for (int k = threadIdx.x; k < 2 * T; k += blockDim.x) {
        const int which = k / T, s = (k % T) / FW, j = k % FW;
        const int cell = which ? next : first;
        loc[which][k % T] = kScale * lam[(size_t)face_of(g, cell, s) * FW + j];
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int row = warp; row < FW; row += 8) {
        // rows of S_K are T = 16N floats (a multiple of four), so every row starts 16-byte aligned
        const float4 *s1 = reinterpret_cast<const float4 *>(S + (size_t)first * T * T + (size_t)((2 * axis + 1) * FW + row) * T);
        const float4 *s2 = reinterpret_cast<const float4 *>(S + (size_t)next * T * T + (size_t)((2 * axis) * FW + row) * T);
        double acc = 0;
#pragma unroll
        for (int t = 0; t < PASSES; ++t) {
            const int j = lane + 32 * t;
            if (j < T4) {
                const float4 a = s1[j], c = s2[j];
                const double *x = loc[0] + 4 * j, *y = loc[1] + 4 * j;
                acc = fma(widen_scaled(a.x), x[0], acc);
                acc = fma(widen_scaled(a.y), x[1], acc);
                acc = fma(widen_scaled(a.z), x[2], acc);
                acc = fma(widen_scaled(a.w), x[3], acc);
                acc = fma(widen_scaled(c.x), y[0], acc);
                acc = fma(widen_scaled(c.y), y[1], acc);
                acc = fma(widen_scaled(c.z), y[2], acc);
                acc = fma(widen_scaled(c.w), y[3], acc);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (lane == 0) {
            const int q = row % N;
            const double d = -face_weight(g, b, face, q) * (speeds[2 * (face * N + q)] + speeds[2 * (face * N + q) + 1]);
            out[(size_t)face * FW + row] = rfma(d, lam[(size_t)face * FW + row], acc);
        }
    }
}
template <int N>
__global__ void __launch_bounds__(256)
k_hdg_apply32(const float *__restrict__ S, const double *__restrict__ speeds, const double *__restrict__ lam,
              double *__restrict__ out, Basis1D b, Grid g) {
    hdg_apply32_body<N>(blockIdx.x, S, speeds, lam, out, b, g);
}
template <int N>
__device__ __forceinline__ void hdg_apply_body(int face, const double *__restrict__ S, const double *__restrict__ speeds,
                                               const double *__restrict__ lam, double *__restrict__ out,
                                               const Basis1D &b, const Grid &g) {
    constexpr int FW = NVAR * N, T = NFACES * FW, T2 = T / 2, PASSES = (T2 + 31) / 32;
    __shared__ __align__(16) double loc[2][T];
    const int axis = face >= g.cells, first = face - axis * g.cells, next = neighbor(g, first, 2 * axis + 1);
    for (int k = threadIdx.x; k < 2 * T; k += blockDim.x) {
        const int which = k / T, s = (k % T) / FW, j = k % FW;
        const int cell = which ? next : first;
        loc[which][k % T] = lam[(size_t)face_of(g, cell, s) * FW + j];
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double2 *l0 = reinterpret_cast<const double2 *>(loc[0]), *l1 = reinterpret_cast<const double2 *>(loc[1]);
    for (int row = warp; row < FW; row += 8) {
        // rows of S_K are T = 16N doubles (an even count), so every row starts 16-byte aligned
        const double2 *s1 = reinterpret_cast<const double2 *>(S + (size_t)first * T * T + (size_t)((2 * axis + 1) * FW + row) * T);
        const double2 *s2 = reinterpret_cast<const double2 *>(S + (size_t)next * T * T + (size_t)((2 * axis) * FW + row) * T);
        double acc = 0;
#pragma unroll
        for (int t = 0; t < PASSES; ++t) {
            const int j = lane + 32 * t;
            if (j < T2) {
                const double2 a = s1[j], b = s2[j], x = l0[j], y = l1[j];
                acc = radd(acc, rfma(a.x, x.x, rfma(a.y, x.y, rfma(b.x, y.x, rmul(b.y, y.y)))));
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (lane == 0) {
            const int q = row % N;
            const double d = -face_weight(g, b, face, q) * (speeds[2 * (face * N + q)] + speeds[2 * (face * N + q) + 1]);
            out[(size_t)face * FW + row] = rfma(d, lam[(size_t)face * FW + row], acc);
        }
    }
}
template <int N>
__global__ void __launch_bounds__(256)
k_hdg_apply(const double *__restrict__ S, const double *__restrict__ speeds, const double *__restrict__ lam,
            double *__restrict__ out, Basis1D b, Grid g) {
    hdg_apply_body<N>(blockIdx.x, S, speeds, lam, out, b, g);
}

// du = -X l_local - y per cell (hybrid.cpp:97-105).
template <int N>
__global__ void __launch_bounds__(256)
k_hdg_recover(const double *__restrict__ X, const double *__restrict__ y, const double *__restrict__ lam,
              double *__restrict__ du, Grid g) {
    constexpr int P = N * N, M = NVAR * P, FW = NVAR * N, T = NFACES * FW;
    __shared__ double loc[T];
    const int cell = blockIdx.x;
    for (int k = threadIdx.x; k < T; k += blockDim.x)
        loc[k] = lam[(size_t)face_of(g, cell, k / FW) * FW + k % FW];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int r = warp; r < M; r += 8) {
        const double *xr = X + (size_t)cell * M * T + (size_t)r * T;
        double acc = 0;
        for (int j = lane; j < T; j += 32) acc += xr[j] * loc[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (lane == 0) du[(size_t)cell * M + r] = -acc - y[(size_t)cell * M + r];
    }
}

// q = -B lambda per cell: the trace coupling column of the condensed cell system
// (hybrid.cpp:35-43: B's column (side, v, q) holds -w tau shape_i at the face line of side),
// so that A^{-1} q - y = -X lambda - y is the recovery of hybrid.cpp:97-105 without X.
template <int N>
__global__ void k_hdg_bmul(const double *__restrict__ lam, const double *__restrict__ speeds, double *__restrict__ out,
                           Basis1D b, Grid g) {
    constexpr int P = N * N, FW = NVAR * N;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)g.cells * P) return;
    const int cell = idx / P, node = idx % P, ix = node % N, iy = node / N;
    double acc[4] = {0, 0, 0, 0};
    for (int side = 0; side < NFACES; ++side) {
        const int face = face_of(g, cell, side);
        const int q = side < 2 ? iy : ix, i = side < 2 ? ix : iy;
        const double ei = (side % 2 ? b.eR : b.eL)[i];
        const double tau = speeds[2 * (face * N + q) + (side % 2 ? 0 : 1)];
        const double stab = face_weight(g, b, face, q) * tau;
#pragma unroll
        for (int v = 0; v < NVAR; ++v) acc[v] += stab * ei * lam[(size_t)face * FW + v * N + q];
    }
#pragma unroll
    for (int v = 0; v < NVAR; ++v) out[(size_t)cell * NVAR * P + v * P + node] = acc[v];
}

// DG residual implied by the Schur error e: -B D^{-1} e lifted into each cell (hybrid.cpp:106-121).
template <int N>
__global__ void k_hdg_recovered_residual(const double *__restrict__ e, const double *__restrict__ speeds,
                                         double *__restrict__ out, Basis1D b, Grid g) {
    constexpr int P = N * N, FW = NVAR * N;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)g.cells * P) return;
    const int cell = idx / P, node = idx % P, ix = node % N, iy = node / N;
    double acc[4] = {0, 0, 0, 0};
    for (int side = 0; side < NFACES; ++side) {
        const int face = face_of(g, cell, side);
        const int q = side < 2 ? iy : ix, i = side < 2 ? ix : iy;
        const double ei = (side % 2 ? b.eR : b.eL)[i];
        const double sa = speeds[2 * (face * N + q)], sb = speeds[2 * (face * N + q) + 1];
        const double w = face_weight(g, b, face, q), d = -w * (sa + sb), tau = side % 2 ? sa : sb;
#pragma unroll
        for (int v = 0; v < NVAR; ++v) acc[v] += ei * (w * tau * e[(size_t)face * FW + v * N + q] / d);
    }
#pragma unroll
    for (int v = 0; v < NVAR; ++v) out[(size_t)cell * NVAR * P + v * P + node] = acc[v];
}

// Projected trace lambda = Phi(U) (discretization.cpp:196-210) from the face restrictions.
template <int N>
__global__ void k_trace_lambda(const double *__restrict__ traces, const double *__restrict__ speeds,
                               double *__restrict__ lam, Grid g) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 2 * g.cells * N) return;
    const int face = idx / N, q = idx % N;
    const int axis = face >= g.cells, cell = face - axis * g.cells;
    const int side = 2 * axis + 1, next = neighbor(g, cell, side);
    const double *Lp = traces + ((size_t)cell * NFACES + side) * N * NVAR + q * NVAR;
    const double *Rp = traces + ((size_t)next * NFACES + side - 1) * N * NVAR + q * NVAR;
    double l[4] = {Lp[0], Lp[1], Lp[2], Lp[3]}, r[4] = {Rp[0], Rp[1], Rp[2], Rp[3]}, fl[4], fr[4];
    flux(g.gamma, l, axis, fl);
    flux(g.gamma, r, axis, fr);
    const double a = speeds[2 * idx], bb = speeds[2 * idx + 1];
#pragma unroll
    for (int v = 0; v < NVAR; ++v)
        lam[(size_t)face * NVAR * N + v * N + q] = (a * l[v] + bb * r[v] + fl[v] - fr[v]) / (a + bb);
}

}  // namespace dgh
