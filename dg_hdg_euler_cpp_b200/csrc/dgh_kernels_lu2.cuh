// Left-looking blocked LU with row partial pivoting on the FP64 tensor pipe (DMMA), one CTA per
// matrix, for the batched DG cell blocks and the HDG condensation.
//
// The right-looking k_lu rewrites the whole trailing matrix after every 32-column panel; with
// hundreds of 0.8-1.2 MB matrices in flight that traffic misses L2 (about 9x the matrix
// size from DRAM) and every column tile costs several CTA barriers.  Here each 32-column panel
// is loaded once into shared memory (all m rows, position order), brought up to date with the
// finished panels to its left (left-looking: for each earlier chunk q, the U rows of the chunk
// by a 32x32 DMMA product with L_qq^{-1}, then the rows below by a DMMA GEMM that reads L from
// the matrix in global memory), factored in shared memory with one CTA barrier per column, and
// written back.  Finished factors are never rewritten, so the matrix is read about
// m/64 times instead of m/16 and written once.
//
// Storage during the factorisation: every row of L and U stays in the ORIGINAL row of the
// matrix (row interchanges only change the position -> row map piv[]), so no data moves on a
// pivot.  For the DG blocks a final pass gathers the rows into position order (the layout
// k_lu_solve expects, then converted to slabs); for the augmented HDG matrix [A | B | r] the
// right-hand-side columns are solved in the same kernel, 32 columns at a time (forward with
// L_qq^{-1}, backward with U_qq^{-1}, both precomputed per panel into a small per-CTA scratch),
// and written as X | y with row i = unknown i, the form k_hdg_schur reads.
//
// Pivoting: the first largest |a| in position order wins ties (LAPACK getrf, Eigen
// PartialPivLU), with LAPACK swap semantics, so the pivot sequence is the reference's.
#pragma once
#include "dgh_kernels_dg.cuh"
#include "dgh_kernels_lu.cuh"

namespace dgh {

// Fused DG mode of k_lu_left (FN = nodes per direction > 0): the kernel walks all cells in one
// persistent launch, assembling each cell's block (k_dg_assemble's entries, collocated volume
// rule) into its CTA's private FP64 slot, factoring it there and writing the reduced-precision
// factors out (FP32 slabs to out32, or FP16 slabs with row scales to out16 / scale16).
struct LLFuse {
    const double *vol = nullptr, *fcache = nullptr, *speeds = nullptr;
    double *slots = nullptr;  // gridDim.x slots of m * m doubles
    __half *out16 = nullptr;
    float *scale16 = nullptr;
    Basis1D b;
    Grid g;
    double inv_step = 0;
    int first = 0;  // cell of block 0 (outputs and perm_out are offset by the caller)
};

constexpr int LL_NB = 32;              // panel width and chunk size
constexpr int LL_AP = 36;              // shared pitch of the panel (= 4 mod 16: conflict-free fragments)
constexpr int LL_THREADS = 256;
constexpr int LL_TRI = 2 * LL_NB * LL_NB;  // doubles of scratch per panel: L_qq^{-1} and U_qq^{-1}

inline size_t lu_left_smem_bytes(int m) {
    const int mp = (m + LL_NB - 1) / LL_NB * LL_NB;
    return sizeof(double) * (size_t)mp * LL_AP + sizeof(int) * (size_t)3 * mp;
}

// One warp-tile step of the chunk product out = T_q * acc[rows q0..q0+31] for the 8 columns
// 8w..8w+7 (warps 0..3), T_q a 32x32 matrix in the scratch (L_qq^{-1} or U_qq^{-1}, padded with
// the identity).  Each warp reads and writes only its own 8 columns.
__device__ __forceinline__ void ll_chunk_tri(double *acc, const double *__restrict__ Tq, int q0) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, lr = lane >> 2, lc = lane & 3;
    if (warp >= 4) return;
    double c[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
#pragma unroll
    for (int kk = 0; kk < LL_NB; kk += 4) {
        const double b = acc[(q0 + kk + lc) * LL_AP + warp * 8 + lr];
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) dmma8x8x4(c[mt], Tq[(mt * 8 + lr) * LL_NB + kk + lc], b);
    }
#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int e = 0; e < 2; ++e) acc[(q0 + mt * 8 + lr) * LL_AP + warp * 8 + 2 * lc + e] = c[mt][e];
}

// acc[rows r in [r_begin, r_end)] -= F(row r, columns q0..q0+qn-1) * acc[rows q0..q0+31], F read
// from the matrix in global memory through piv (F = L below the chunk, U above it).  16-row
// blocks are dealt round-robin to the 8 warps; each warp holds 2 x 4 DMMA tiles.
__device__ __forceinline__ void ll_chunk_gemm(double *acc, const double *__restrict__ A, int ld, const int *piv,
                                              int q0, int qn, int r_begin, int r_end) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, lr = lane >> 2, lc = lane & 3;
    const int R = r_end - r_begin;
    for (int blk = warp; blk * 16 < R; blk += LL_THREADS / 32) {
        const int rb = r_begin + blk * 16;
        double c[2][4][2];
        const double *frow[2];
        bool valid[2];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const int r = rb + mt * 8 + lr;
            valid[mt] = r < r_end;
            frow[mt] = A + (size_t)(valid[mt] ? piv[r] : 0) * ld + q0;
#pragma unroll
            for (int nt = 0; nt < 4; ++nt)
#pragma unroll
                for (int e = 0; e < 2; ++e) c[mt][nt][e] = valid[mt] ? acc[r * LL_AP + nt * 8 + 2 * lc + e] : 0.;
        }
        if (qn == LL_NB) {  // full chunk: every operand load of the block issued up front
            double a[2][LL_NB / 4];
#pragma unroll
            for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                for (int k = 0; k < LL_NB / 4; ++k) a[mt][k] = valid[mt] ? -__ldg(frow[mt] + 4 * k + lc) : 0.;
#pragma unroll
            for (int k = 0; k < LL_NB / 4; ++k) {
                double b[4];
#pragma unroll
                for (int nt = 0; nt < 4; ++nt) b[nt] = acc[(q0 + 4 * k + lc) * LL_AP + nt * 8 + lr];
#pragma unroll
                for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                    for (int nt = 0; nt < 4; ++nt) dmma8x8x4(c[mt][nt], a[mt][k], b[nt]);
            }
        } else {
            for (int kk = 0; kk < qn; kk += 4) {
                double a[2], b[4];
#pragma unroll
                for (int mt = 0; mt < 2; ++mt) a[mt] = valid[mt] ? -__ldg(frow[mt] + kk + lc) : 0.;
#pragma unroll
                for (int nt = 0; nt < 4; ++nt) b[nt] = acc[(q0 + kk + lc) * LL_AP + nt * 8 + lr];
#pragma unroll
                for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                    for (int nt = 0; nt < 4; ++nt) dmma8x8x4(c[mt][nt], a[mt], b[nt]);
            }
        }
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            if (!valid[mt]) continue;
            const int r = rb + mt * 8 + lr;
#pragma unroll
            for (int nt = 0; nt < 4; ++nt)
#pragma unroll
                for (int e = 0; e < 2; ++e) acc[r * LL_AP + nt * 8 + 2 * lc + e] = c[mt][nt][e];
        }
    }
}

// acc[i][c] = A[piv[i]][j0 + c] for positions i < m and c < ncols, zero elsewhere (rows < mp,
// columns < 32); eight independent loads in flight per thread.
__device__ __forceinline__ void ll_load_cols(double *acc, const double *__restrict__ A, int ld, const int *piv, int m,
                                             int mp, int j0, int ncols) {
    constexpr int U = 8;
    const int total = mp * LL_NB;
    for (int base = threadIdx.x; base < total; base += U * LL_THREADS) {
        double v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int idx = base + u * LL_THREADS, i = idx / LL_NB, cc = idx % LL_NB;
            v[u] = (idx < total && i < m && cc < ncols) ? __ldg(A + (size_t)piv[i] * ld + j0 + cc) : 0.;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int idx = base + u * LL_THREADS;
            if (idx < total) acc[(idx / LL_NB) * LL_AP + idx % LL_NB] = v[u];
        }
    }
}

// Asks L2 for the rows [r_begin, r_end) x columns q0..q0+31 of the matrix (through piv), the
// operand of the next chunk product, so that its loads find L2 instead of DRAM.
__device__ __forceinline__ void ll_prefetch(const double *__restrict__ A, int ld, const int *piv, int q0,
                                            int r_begin, int r_end) {
    for (int idx = threadIdx.x; idx < 3 * (r_end - r_begin); idx += LL_THREADS) {
        const int r = r_begin + idx / 3, part = idx % 3;
        const char *p = reinterpret_cast<const char *>(A + (size_t)piv[r] * ld + q0) + (part == 2 ? 255 : 128 * part);
        asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
    }
}

// Pitch (doubles) of the 32-row staging area of the final layout passes: >= m and = 2 mod 16,
// so that lanes reading 16 bytes of consecutive rows hit distinct banks.  32 * pitch doubles fit
// the panel area of mp * LL_AP for every m = 4 n^2 the kernel accepts (n <= 11).
__device__ __forceinline__ int ll_stage_pitch(int m) { return m + (18 - m % 16) % 16; }

// dst[0..m) = src[0..m) by one warp: 16-byte loads, up to four in flight per lane (m even and
// both rows 16-byte aligned: every row starts at a multiple of 8 m bytes, m = 4 n^2).
__device__ __forceinline__ void ll_stage_row(double *dst, const double *src, int m) {
    const int lane = threadIdx.x & 31, h = m / 2;
    const double2 *s2 = reinterpret_cast<const double2 *>(src);
    double2 *d2 = reinterpret_cast<double2 *>(dst);
    for (int c0 = lane; c0 < h; c0 += 4 * 32) {
        double2 v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int c = c0 + 32 * u;
            if (c < h) v[u] = s2[c];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int c = c0 + 32 * u;
            if (c < h) d2[c] = v[u];
        }
    }
}

// Warp-wide pivot choice over the lanes' candidates (v, position, slot): the largest v wins,
// then the smallest position (v = |a|, -1 for a NaN entry, -2 for no candidate).  v maps to an
// order-preserving 64-bit key (non-negative doubles order as their bit patterns; -0 is folded
// to +0, which compares equal to it), reduced as two 32-bit halves with redux.sync; the winner's
// own (v, position, slot) are then broadcast, so every lane ends with the value the pairwise
// comparison would have kept.
__device__ __forceinline__ void ll_warp_argmax(double &bv, int &bp, int &bs) {
    const unsigned long long key = bv == -2. ? 0ull
                                   : bv == -1. ? 1ull
                                               : (unsigned long long)__double_as_longlong(fabs(bv)) + 2ull;
    const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
    const unsigned mh = __reduce_max_sync(0xffffffffu, hi);
    const unsigned ml = __reduce_max_sync(0xffffffffu, hi == mh ? lo : 0u);
    const bool top = hi == mh && lo == ml;
    const unsigned mpos = __reduce_min_sync(0xffffffffu, top ? (unsigned)bp : 0xffffffffu);
    const int src = __ffs(__ballot_sync(0xffffffffu, top && (unsigned)bp == mpos)) - 1;
    bv = __shfl_sync(0xffffffffu, bv, src);
    bp = __shfl_sync(0xffffffffu, bp, src);
    bs = __shfl_sync(0xffffffffu, bs, src);
}

// Batched LU.  AUG = false: pool holds m x m blocks (ld = m); on exit row i of each block is
// position i of the factors (unit L below, U on and above the diagonal), perm_out[i] = its
// original row, and with slab_out the block is rewritten in the slab layout of k_lu_solve.
// With out32 != nullptr the factors are instead written, rounded to FP32, in the FP32 slab
// layout to out32 (m x m per block) and pool is left in original-row order: the mixed
// precision preconditioner factors in FP64 and stores FP32.
// AUG = true: pool holds [A | B | r] with ld > m; on exit X | y = A^{-1}[B r] (row i = unknown i)
// is in columns m..ld-1, or, with x_out, in x_out (m x (ld - m - 1) row-major per matrix) and
// y_out (m per matrix); the A part holds the factors in original-row order (not used later).
// tri: per-CTA scratch of ceil(m/32) * LL_TRI doubles.
template <bool AUG, int FN = 0>
__global__ void __launch_bounds__(LL_THREADS, 2)
k_lu_left(double *__restrict__ pool, size_t stride, int m, int ld, int count, double *__restrict__ tri_all,
          int *__restrict__ perm_out, int *status, int singular_bit, int slab_out, float *__restrict__ out32,
          double *__restrict__ x_out, double *__restrict__ y_out, LLFuse fu = LLFuse()) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const int mp = (m + LL_NB - 1) / LL_NB * LL_NB, P = mp / LL_NB;
    double *acc = reinterpret_cast<double *>(smraw);  // mp rows x LL_AP
    int *piv = reinterpret_cast<int *>(acc + (size_t)mp * LL_AP);
    int *posmap = piv + mp;   // slot -> position after a panel
    int *slotof = posmap + mp;  // position -> slot (the panel's first nb positions) / scratch
    __shared__ double cand_v[2][LL_THREADS / 32];
    __shared__ int cand_p[2][LL_THREADS / 32], cand_s[2][LL_THREADS / 32];
    __shared__ int bad;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = LL_THREADS / 32;
    double *tri = tri_all + (size_t)blockIdx.x * P * LL_TRI;

    __shared__ Basis1D fsb;
    if constexpr (FN > 0) stage_basis<FN>(fu.b, fsb);
    for (int blk = blockIdx.x; blk < count; blk += gridDim.x) {
        double *A = pool + (size_t)blk * stride;
        if constexpr (FN > 0) {
            // assemble the cell's block into this CTA's slot (tables in the panel area)
            constexpr int FP = FN * FN, FM = NVAR * FP;
            A = fu.slots + (size_t)blockIdx.x * FM * FM;
            double *jx = acc, *jy = jx + FP * 16, *fj = jy + FP * 16;
            __syncthreads();
            cell_tables<FN, false>(fu.first + blk, fu.vol, fu.fcache, fu.speeds, fsb, fu.g, jx, jy, fj);
            __syncthreads();
            for (int idx = tid; idx < FM * FM; idx += LL_THREADS)
                A[idx] = cell_block_entry<FN>(idx / FM, idx % FM, jx, jy, fj, fsb, fu.g, fu.inv_step, true);
            __syncthreads();
        }
        for (int i = tid; i < mp; i += LL_THREADS) piv[i] = i < m ? i : 0;
        if (tid == 0) bad = 0;
        __syncthreads();

        for (int p = 0; p < P; ++p) {
            const int k0 = p * LL_NB, nb = min(LL_NB, m - k0);
            // ---- load panel columns k0..k0+nb-1 of every position (zero padding)
            ll_load_cols(acc, A, ld, piv, m, mp, k0, nb);
            __syncthreads();
            // ---- left-looking update with the finished chunks
            for (int q = 0; q < p; ++q) {
                const int q0 = q * LL_NB;
                if (q + 1 < p) ll_prefetch(A, ld, piv, q0 + LL_NB, q0 + 2 * LL_NB, m);
                ll_chunk_tri(acc, tri + (size_t)q * LL_TRI, q0);
                __syncthreads();
                ll_chunk_gemm(acc, A, ld, piv, q0, LL_NB, q0 + LL_NB, m);
                __syncthreads();
            }
            // ---- factor the panel: rows at positions k0..m-1, one barrier per column.  Slot s
            // is acc row s.  The rows come in groups of 8 dealt round-robin to the warps (group G
            // to warp G % 8), so every warp holds about (m - k0) / 8 rows; lane l owns the slots
            // s0 (group 8 * (l / 8) + warp, row l % 8) and s1 = s0 + 256 and tracks their positions
            // (LAPACK swaps).  A warp both eliminates and searches its own rows, so only the pivot
            // choice crosses warps (one barrier per column).
            const int s0 = k0 + 8 * warp + 64 * (lane >> 3) + (lane & 7), s1 = s0 + LL_THREADS;
            int pos0 = s0, pos1 = s1;
            // Sub-panels of 4 columns: inside a sub-panel each column updates only the sub-panel's
            // later columns; after its 4 columns, the warp's unpivoted rows get the rank-4 update
            // of the panel's remaining columns on the tensor pipe (pivoted rows have a zero operand
            // row, so they are left alone).  U of the sub-panel's pivot rows (the 4 x 4 unit-lower
            // solve of their raw remaining columns) is written back by warp 0 one sub-panel later,
            // when no warp reads the raw values any more.
            const int r8 = lane >> 2, g4 = lane & 3;
            int ppsl[4] = {0, 0, 0, 0}, pb0 = -1;
            // u_k(col) for the 4 pivot rows of a sub-panel starting at column c0
            auto sub_u = [&](const int (&ps)[4], int c0, int col, double (&u)[4]) {
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const double *pr = acc + ps[k] * LL_AP;
                    double v = pr[col];
#pragma unroll
                    for (int j = 0; j < k; ++j) v -= pr[c0 + j] * u[j];
                    u[k] = v;
                }
            };
            for (int b0 = 0; b0 < nb; b0 += 4) {
                int psl[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int jj = b0 + u, tp = k0 + jj;
                    double bv = -2.;
                    int bp = 0x7fffffff, bs = -1;
                    auto consider = [&](int s, int ps) {
                        if (s >= m || ps < tp) return;
                        const double a = acc[s * LL_AP + jj];
                        double v = a < 0 ? -a : a;
                        if (!(v == v)) v = -1.;  // a NaN row is chosen only if nothing else is left
                        if (v > bv || (v == bv && ps < bp)) { bv = v; bp = ps; bs = s; }
                    };
                    consider(s0, pos0);
                    consider(s1, pos1);
                    ll_warp_argmax(bv, bp, bs);
                    if (lane == 0) {
                        cand_v[jj & 1][warp] = bv;
                        cand_p[jj & 1][warp] = bp;
                        cand_s[jj & 1][warp] = bs;
                    }
                    __syncthreads();
                    bv = cand_v[jj & 1][0];
                    bp = cand_p[jj & 1][0];
                    bs = cand_s[jj & 1][0];
#pragma unroll
                    for (int w = 1; w < NW; ++w) {
                        const double ov = cand_v[jj & 1][w];
                        const int op = cand_p[jj & 1][w];
                        if (ov > bv || (ov == bv && op < bp)) { bv = ov; bp = op; bs = cand_s[jj & 1][w]; }
                    }
                    psl[u] = bs;
                    // swap positions tp and bp (the slot at tp moves to bp)
                    if (s0 < m) { if (s0 == bs) pos0 = tp; else if (pos0 == tp) pos0 = bp; }
                    if (s1 < m) { if (s1 == bs) pos1 = tp; else if (pos1 == tp) pos1 = bp; }
                    if (u == 0 && pb0 >= 0 && warp == 0) {  // U of the previous sub-panel's pivot rows
                        const int col = pb0 + 4 + lane;
                        if (col < nb) {
                            double uu[4];
                            sub_u(ppsl, pb0, col, uu);
#pragma unroll
                            for (int k = 0; k < 4; ++k) acc[ppsl[k] * LL_AP + col] = uu[k];
                        }
                    }
                    const double *prow = acc + bs * LL_AP;
                    const double pv = prow[jj], rpv = pv != 0. ? 1. / pv : 1.;
                    const int cme = b0 + g4;  // this lane's column inside the sub-panel
                    const double pcm = prow[cme];
                    // elimination inside the sub-panel, 8 rows at a time: lane = (row r8, column b0+g4).
                    // Group grp of batch t holds the slots of lanes 8 grp .. 8 grp + 7 (s0 for t = 0,
                    // s1 for t = 1), so the rows still below the pivot are bits of two ballots.  All
                    // multipliers are read first, then the sub-panel columns updated, then the
                    // multipliers stored over column jj once every lane has read it.
                    const unsigned own0 = __ballot_sync(0xffffffffu, s0 < m && pos0 > tp);
                    const unsigned own1 = __ballot_sync(0xffffffffu, s1 < m && pos1 > tp);
                    double lv[2][4];
#pragma unroll
                    for (int t = 0; t < 2; ++t)
#pragma unroll
                        for (int grp = 0; grp < 4; ++grp) {
                            const bool act = ((t ? own1 : own0) >> (8 * grp + r8)) & 1u;
                            const double *row = acc + min(k0 + 8 * warp + t * LL_THREADS + 64 * grp + r8, mp - 1) * LL_AP;
                            lv[t][grp] = act ? row[jj] * rpv : 0.;
                        }
#pragma unroll
                    for (int t = 0; t < 2; ++t)
#pragma unroll
                        for (int grp = 0; grp < 4; ++grp) {
                            const bool act = ((t ? own1 : own0) >> (8 * grp + r8)) & 1u;
                            double *row = acc + min(k0 + 8 * warp + t * LL_THREADS + 64 * grp + r8, mp - 1) * LL_AP;
                            if (act && cme > jj) row[cme] -= lv[t][grp] * pcm;
                        }
                    __syncwarp();
#pragma unroll
                    for (int t = 0; t < 2; ++t)
#pragma unroll
                        for (int grp = 0; grp < 4; ++grp) {
                            const bool act = ((t ? own1 : own0) >> (8 * grp + r8)) & 1u;
                            double *row = acc + min(k0 + 8 * warp + t * LL_THREADS + 64 * grp + r8, mp - 1) * LL_AP;
                            if (act && g4 == 0) row[jj] = lv[t][grp];
                        }
                    __syncwarp();
                }
                // rank-4 update of columns b0+4..nb-1 for this warp's unpivoted rows
                if (b0 + 4 < nb) {
                    const int tp = k0 + b0 + 3;
                    double bfr[4];
#pragma unroll
                    for (int nt = 0; nt < 4; ++nt) {
                        const int col = b0 + 4 + 8 * nt + r8;
                        bfr[nt] = 0.;
                        if (col < nb) {
                            double uu[4];
                            sub_u(psl, b0, col, uu);
                            bfr[nt] = g4 == 0 ? uu[0] : g4 == 1 ? uu[1] : g4 == 2 ? uu[2] : uu[3];
                        }
                    }
                    const unsigned own0 = __ballot_sync(0xffffffffu, s0 < m && pos0 > tp);
                    const unsigned own1 = __ballot_sync(0xffffffffu, s1 < m && pos1 > tp);
#pragma unroll
                    for (int t = 0; t < 2; ++t) {
                        const int sb = k0 + 8 * warp + t * LL_THREADS;
#pragma unroll
                        for (int grp = 0; grp < 4; ++grp) {
                            const unsigned gbits = ((t ? own1 : own0) >> (8 * grp)) & 0xffu;
                            if (!gbits) continue;  // warp-uniform: no row of the group below the pivots
                            const bool act = (gbits >> r8) & 1u;
                            double *row = acc + min(sb + 64 * grp + r8, mp - 1) * LL_AP;  // used only if act
                            const double a = act ? -row[b0 + g4] : 0.;
#pragma unroll
                            for (int nt = 0; nt < 4; ++nt) {
                                if (b0 + 4 + 8 * nt >= nb) break;
                                double c[2];
#pragma unroll
                                for (int e = 0; e < 2; ++e) {
                                    const int col = b0 + 4 + 8 * nt + 2 * g4 + e;
                                    c[e] = (act && col < nb) ? row[col] : 0.;
                                }
                                dmma8x8x4(c, a, bfr[nt]);
#pragma unroll
                                for (int e = 0; e < 2; ++e) {
                                    const int col = b0 + 4 + 8 * nt + 2 * g4 + e;
                                    if (act && col < nb) row[col] = c[e];
                                }
                            }
                        }
                    }
                    __syncwarp();
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) ppsl[k] = psl[k];
                pb0 = b0;
            }
            // ---- new positions, write back, permutation update
            if (s0 < m) posmap[s0] = pos0;
            if (s1 < m) posmap[s1] = pos1;
            __syncthreads();
            for (int s = k0 + tid; s < m; s += LL_THREADS)
                if (posmap[s] < k0 + nb) slotof[posmap[s] - k0] = s;
            for (int idx = tid; idx < m * LL_NB; idx += LL_THREADS) {
                const int s = idx / LL_NB, cc = idx % LL_NB;
                if (cc < nb) A[(size_t)piv[s] * ld + k0 + cc] = acc[s * LL_AP + cc];
            }
            __syncthreads();
            // L_pp^{-1} (unit lower) by columns: thread c < 32; U_pp^{-1} (upper) by thread 32 + c.
            // Each column is built in registers (fully unrolled), then stored (identity padding).
            {
                double *Li = tri + (size_t)p * LL_TRI, *Ui = Li + LL_NB * LL_NB;
                if (tid < LL_NB) {
                    const int cc = tid;
                    double col[LL_NB];
#pragma unroll
                    for (int i = 0; i < LL_NB; ++i) {
                        double v = i == cc ? 1. : 0.;
                        if (i < nb && cc < nb && i > cc) {
                            const double *row = acc + slotof[i] * LL_AP;
                            double sum = 0;
#pragma unroll
                            for (int l = 0; l < i; ++l)
                                if (l >= cc) sum += row[l] * col[l];
                            v = -sum;
                        }
                        col[i] = v;
                    }
#pragma unroll
                    for (int i = 0; i < LL_NB; ++i) Li[i * LL_NB + cc] = col[i];
                } else if (AUG && tid < 2 * LL_NB) {
                    const int cc = tid - LL_NB;
                    double col[LL_NB];
#pragma unroll
                    for (int i = LL_NB - 1; i >= 0; --i) {
                        double v = i == cc ? 1. : 0.;
                        if (i < nb && cc < nb && i <= cc) {
                            const double *row = acc + slotof[i] * LL_AP;
                            double sum = i == cc ? 1. : 0.;
#pragma unroll
                            for (int l = i + 1; l < LL_NB; ++l)
                                if (l <= cc) sum -= row[l] * col[l];
                            v = sum / row[i];
                        }
                        col[i] = v;
                    }
#pragma unroll
                    for (int i = 0; i < LL_NB; ++i) Ui[i * LL_NB + cc] = col[i];
                } else if (tid >= 64 && tid < 64 + LL_NB && tid - 64 < nb) {
                    const double d = acc[slotof[tid - 64] * LL_AP + (tid - 64)];
                    if (!isfinite(d) || !(fabs(d) > 2.2250738585072014e-308)) bad = 1;
                }
            }
            __syncthreads();  // the inverses above read slotof[0..nb)
            for (int s = k0 + tid; s < m; s += LL_THREADS) slotof[posmap[s]] = piv[s];  // position -> row
            __syncthreads();
            for (int i = k0 + tid; i < m; i += LL_THREADS) piv[i] = slotof[i];
            __syncthreads();
        }

        if (AUG) {
            if (perm_out)  // the factors stay in original-row order: position i is row piv[i]
                for (int i = tid; i < m; i += LL_THREADS) perm_out[(size_t)blk * m + i] = piv[i];
            // ---- right-hand sides: forward with L, backward with U, 32 columns at a time
            for (int j0 = m; j0 < ld; j0 += LL_NB) {
                const int ncols = min(LL_NB, ld - j0);
                ll_load_cols(acc, A, ld, piv, m, mp, j0, ncols);
                __syncthreads();
                for (int q = 0; q < P; ++q) {
                    const int q0 = q * LL_NB;
                    if (q0 + 2 * LL_NB < m) ll_prefetch(A, ld, piv, q0 + LL_NB, q0 + 2 * LL_NB, m);
                    ll_chunk_tri(acc, tri + (size_t)q * LL_TRI, q0);
                    __syncthreads();
                    if (q0 + LL_NB < m) {
                        ll_chunk_gemm(acc, A, ld, piv, q0, LL_NB, q0 + LL_NB, m);
                        __syncthreads();
                    }
                }
                for (int q = P - 1; q >= 0; --q) {
                    const int q0 = q * LL_NB, qn = min(LL_NB, m - q0);
                    if (q >= 2) ll_prefetch(A, ld, piv, q0 - LL_NB, 0, q0 - LL_NB);
                    ll_chunk_tri(acc, tri + (size_t)q * LL_TRI + LL_NB * LL_NB, q0);
                    __syncthreads();
                    if (q0 > 0) {
                        ll_chunk_gemm(acc, A, ld, piv, q0, qn, 0, q0);
                        __syncthreads();
                    }
                }
                const int T = ld - m - 1;
                for (int idx = tid; idx < m * LL_NB; idx += LL_THREADS) {
                    const int i = idx / LL_NB, cc = idx % LL_NB, col = j0 + cc - m;
                    if (cc >= ncols) continue;
                    const double v = acc[i * LL_AP + cc];
                    if (!x_out) A[(size_t)i * ld + j0 + cc] = v;
                    else if (col < T) x_out[(size_t)blk * m * T + (size_t)i * T + col] = v;
                    else y_out[(size_t)blk * m + i] = v;
                }
                __syncthreads();
            }
        } else if (FN > 0 && fu.out16) {
            // ---- FP16 slabs with row scales (k_pack_half's layout) from the original-row storage:
            // stage 32 position rows, each row's largest |U| by a warp, then 8-column groups
            const int sp = ll_stage_pitch(m), mp8 = pad8(m);
            double *stage = acc;
            __shared__ float rsc[32];
            __half *out = fu.out16 + (size_t)blk * m * mp8;
            for (int r0 = 0; r0 < m; r0 += 32) {
                const int nt = min(32, m - r0);
                for (int rr = warp; rr < nt; rr += NW) ll_stage_row(stage + (size_t)rr * sp, A + (size_t)piv[r0 + rr] * ld, m);
                __syncthreads();
                for (int rr = warp; rr < nt; rr += NW) {
                    double big = 0;
                    for (int j = r0 + rr + lane; j < m; j += 32) big = fmax(big, fabs(stage[(size_t)rr * sp + j]));
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) big = fmax(big, __shfl_xor_sync(0xffffffffu, big, o));
                    if (lane == 0) {
                        rsc[rr] = big > 0 ? (float)(1. / big) : 1.f;
                        fu.scale16[(size_t)blk * m + r0 + rr] = rsc[rr];
                    }
                }
                __syncthreads();
                for (int gg = warp; gg < mp8 / H_W; gg += NW)
                    for (int rr = lane; rr < nt; rr += 32) {
                        __align__(16) __half v[H_W];
                        const double inv = (double)rsc[rr];
#pragma unroll
                        for (int w = 0; w < H_W; ++w) {
                            const int j = gg * H_W + w;
                            const double a = j < m ? stage[(size_t)rr * sp + j] : 0.;
                            v[w] = __double2half(j >= r0 + rr ? a * inv : a);
                        }
                        *reinterpret_cast<uint4 *>(out + (size_t)r0 * mp8 + (size_t)gg * nt * H_W + rr * H_W) =
                            *reinterpret_cast<const uint4 *>(v);
                    }
                __syncthreads();
            }
            for (int i = tid; i < m; i += LL_THREADS) perm_out[(size_t)blk * m + i] = piv[i];
        } else if (out32) {
            // ---- FP32 slabs straight from the original-row storage: stage 32 position rows
            // (16-byte loads, several in flight per thread), then each lane converts one row's
            // 4 columns of a slab group into one float4
            constexpr int W = SlabVec<float>::W;
            const int sp = ll_stage_pitch(m);
            double *stage = acc;
            float4 *out = reinterpret_cast<float4 *>(out32 + (size_t)blk * m * m);
            for (int r0 = 0; r0 < m; r0 += 32) {
                const int nt = min(32, m - r0);
                for (int rr = warp; rr < nt; rr += NW) ll_stage_row(stage + (size_t)rr * sp, A + (size_t)piv[r0 + rr] * ld, m);
                __syncthreads();
                float4 *reg = out + (size_t)r0 * m / W;
                for (int g = warp; g < m / W; g += NW)
                    for (int rr = lane; rr < nt; rr += 32) {
                        const double2 a = *reinterpret_cast<const double2 *>(stage + (size_t)rr * sp + g * W);
                        const double2 b = *reinterpret_cast<const double2 *>(stage + (size_t)rr * sp + g * W + 2);
                        reg[(size_t)g * nt + rr] = make_float4((float)a.x, (float)a.y, (float)b.x, (float)b.y);
                    }
                __syncthreads();
            }
            for (int i = tid; i < m; i += LL_THREADS) perm_out[(size_t)blk * m + i] = piv[i];
        } else {
            // ---- gather the rows into position order, 32 columns at a time
            for (int c0 = 0; c0 < m; c0 += LL_NB) {
                const int w = min(LL_NB, m - c0);
                ll_load_cols(acc, A, ld, piv, m, mp, c0, w);
                __syncthreads();
                for (int idx = tid; idx < m * LL_NB; idx += LL_THREADS) {
                    const int i = idx / LL_NB, cc = idx % LL_NB;
                    if (cc < w) A[(size_t)i * ld + c0 + cc] = acc[i * LL_AP + cc];
                }
                __syncthreads();
            }
            for (int i = tid; i < m; i += LL_THREADS) perm_out[(size_t)blk * m + i] = piv[i];
            if (slab_out) {  // in-place conversion to the slab layout read by k_lu_solve
                constexpr int W = SlabVec<double>::W;
                const int sp = ll_stage_pitch(m);
                double *stage = acc;
                for (int r0 = 0; r0 < m; r0 += 32) {
                    const int nt = min(32, m - r0);
                    double *reg = A + (size_t)r0 * m;
                    for (int rr = warp; rr < nt; rr += NW) ll_stage_row(stage + (size_t)rr * sp, reg + (size_t)rr * m, m);
                    __syncthreads();
                    double2 *reg2 = reinterpret_cast<double2 *>(reg);
                    for (int g = warp; g < m / W; g += NW)
                        for (int rr = lane; rr < nt; rr += 32)
                            reg2[(size_t)g * nt + rr] = *reinterpret_cast<const double2 *>(stage + (size_t)rr * sp + g * W);
                    __syncthreads();
                }
            }
        }
        if (tid == 0 && bad) atomicOr(status, singular_bit);
        __syncthreads();
    }
}

}  // namespace dgh
