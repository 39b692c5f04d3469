// Lockstep batch of GMRES solves (no counterpart in the reference): the restart cycles of many
// independent DG Newton systems, or of many condensed HDG Schur systems, of any degree and mesh
// size, advanced together, each phase of an Arnoldi step one kernel launch over all members
// (the operator once per degree present, the block-Jacobi preconditioner once per factor
// layout present).  A launch's CTAs are split into
// per-member ranges; each CTA finds its member in the table and runs the single-problem kernel
// body on that member's own buffers with that member's own block partition, so every member's
// numbers are bitwise those of its single-problem solve (gmres.cpp:17-86, same kernels).
#pragma once
#include "dgh_kernels_dg.cuh"
#include "dgh_kernels_hdg.cuh"
#include "dgh_kernels_krylov.cuh"
#include "dgh_kernels_lu.cuh"

namespace dgh {

// One member: its context's GMRES state and vectors, its block-Jacobi factors, its operator's
// data and the first CTA of each batched launch it takes part in.  A DG member (operator J)
// carries its cell-block factors and J·v caches; an HDG member (the condensed Schur operator)
// carries its face-block factors or FP32 inverses in the same fields (m = fw, cells = faces)
// and its Schur blocks S (FP64, or FP32 with c32).
struct LsMember {
    GmresDev *gdev;
    double *V, *w, *z, *red, *partial, *coef, *x, *rhs, *r;
    const double *W;
    size_t ld;
    long long n;
    int red0, red_blocks;  // CTAs of the batched sweeps and reductions (red_blocks = the member's red_grid)
    int live;              // 1 while the member's GMRES runs (host-set per restart cycle)
    // block-Jacobi factors (FP64 / FP32 slabs, or FP16 slabs with row scales)
    const void *pool;
    const float *scale;
    const int *perm;
    size_t stride;
    int m, cells;
    int solve0;  // first CTA in the batched solve of its factor layout
    // J·v (collocated DG operator)
    double *traces;
    const double *vol, *fcache, *speeds;
    const Basis1D *basis;
    Grid g;
    double inv_step;
    int team0;  // first CTA in the batched operator launch of its degree (J·v: cell teams; Schur: faces)
    // condensed Schur operator (HDG members)
    const void *S;
    int c32;
};

// vector selectors of the batched kernels
enum LsVec { LS_Z = 0, LS_W = 1, LS_X = 2, LS_R = 3, LS_RHS = 4, LS_VJ = 5, LS_VJ1 = 6 };
__device__ __forceinline__ double *ls_vec(const LsMember &t, int sel, int j) {
    switch (sel) {
        case LS_Z: return t.z;
        case LS_W: return t.w;
        case LS_X: return t.x;
        case LS_R: return t.r;
        case LS_RHS: return t.rhs;
        case LS_VJ: return t.V + (size_t)j * t.ld;
        default: return t.V + (size_t)(j + 1) * t.ld;
    }
}
// gate: 0 = the member's cycle is live (start and finish segments); 1 = live and its current
// Arnoldi step continues (the device flag the previous step set)
__device__ __forceinline__ bool ls_on(const LsMember &t, int gate) { return t.live && (gate == 0 || t.gdev->cont); }

// The member of table entries [first, first + count) whose CTA range (offset `field`) holds bx.
enum LsRange { LS_RED = 0, LS_SOLVE = 1, LS_TEAM = 2 };
__device__ __forceinline__ int ls_start(const LsMember &t, int field) {
    return field == LS_RED ? t.red0 : field == LS_SOLVE ? t.solve0 : t.team0;
}
__device__ __forceinline__ int ls_find(const LsMember *t, int first, int count, int bx, int field) {
    int i = first;
    while (i + 1 < first + count && bx >= ls_start(t[i + 1], field)) ++i;
    return i;
}

// ---- the CGS2 sweeps, norms and reductions ---------------------------------------------------
template <int NV>
__global__ void __launch_bounds__(KR_THREADS) k_ls_mdot(const LsMember *t, int count, int K) {
    const LsMember &a = t[ls_find(t, 0, count, blockIdx.x, LS_RED)];
    if (!ls_on(a, 1)) return;
    mdot_body<NV>(blockIdx.x - a.red0, a.red_blocks, a.V, a.ld, K, a.w, a.W, a.n, a.partial);
}
template <int NV, int MODE>
__global__ void __launch_bounds__(KR_THREADS) k_ls_maxpy(const LsMember *t, int count, int K) {
    const LsMember &a = t[ls_find(t, 0, count, blockIdx.x, LS_RED)];
    if (!ls_on(a, 1)) return;
    maxpy_body<NV, MODE>(blockIdx.x - a.red0, a.red_blocks, a.V, a.ld, K, MODE == 0 ? a.red : a.red + KR_MAXK, a.w,
                         a.W, a.n, a.partial);
}
// out = red (which 0), red + KR_MAXK (1), red + 2 KR_MAXK (2) or the cycle's final |r|^2 (3);
// CTA i K + k reduces entry k of member i
__global__ void __launch_bounds__(KR_THREADS) k_ls_reduce(const LsMember *t, int count, int K, int which, int gate) {
    const LsMember &a = t[blockIdx.x / K];
    if (!ls_on(a, gate)) return;
    double *out = which == 3 ? &a.gdev->rnorm2 : a.red + which * KR_MAXK;
    reduce_body(blockIdx.x % K, a.partial, a.red_blocks, out);
}
__global__ void __launch_bounds__(KR_THREADS) k_ls_wnorm2(const LsMember *t, int count) {
    const LsMember &a = t[ls_find(t, 0, count, blockIdx.x, LS_RED)];
    if (!ls_on(a, 0)) return;
    wnorm2_body(blockIdx.x - a.red0, a.red_blocks, a.r, a.W, 0, a.n, a.partial);
}
// dst = src / sqrt(red[2 KR_MAXK])
__global__ void __launch_bounds__(KR_THREADS) k_ls_scale_div(const LsMember *t, int count, int src, int dst, int j,
                                                             int gate) {
    const LsMember &a = t[ls_find(t, 0, count, blockIdx.x, LS_RED)];
    if (!ls_on(a, gate)) return;
    scale_div_body(blockIdx.x - a.red0, a.red_blocks, ls_vec(a, src, j), a.red + 2 * KR_MAXK, 1, ls_vec(a, dst, j), a.n);
}
// out = ca x + cb y over the selected vectors (live members)
__global__ void __launch_bounds__(KR_THREADS) k_ls_axpby(const LsMember *t, int count, double ca, int x, double cb,
                                                         int y, int out) {
    const LsMember &a = t[ls_find(t, 0, count, blockIdx.x, LS_RED)];
    if (!ls_on(a, 0)) return;
    axpby_body(blockIdx.x - a.red0, a.red_blocks, ca, ls_vec(a, x, 0), cb, ls_vec(a, y, 0), ls_vec(a, out, 0), a.n);
}
// w = V y (the cycle's correction direction)
__global__ void __launch_bounds__(KR_THREADS) k_ls_lincomb(const LsMember *t, int count) {
    const LsMember &a = t[ls_find(t, 0, count, blockIdx.x, LS_RED)];
    if (!ls_on(a, 0)) return;
    lincomb_dyn_body(blockIdx.x - a.red0, a.red_blocks, a.V, a.ld, &a.gdev->count, a.coef, a.w, a.n);
}

// ---- GMRES control, one CTA per member ---------------------------------------------------------
__global__ void k_ls_gmres_init(const LsMember *t) {
    const LsMember &a = t[blockIdx.x];
    if (threadIdx.x == 0 && ls_on(a, 0)) gmres_init_body(a.gdev, a.red + 2 * KR_MAXK);
}
__global__ void k_ls_gmres_update(const LsMember *t, int j) {
    const LsMember &a = t[blockIdx.x];
    if (threadIdx.x == 0 && ls_on(a, 1)) gmres_update_body(a.gdev, a.red, j);
}
__global__ void k_ls_gmres_backsolve(const LsMember *t) {
    const LsMember &a = t[blockIdx.x];
    if (threadIdx.x == 0 && ls_on(a, 0)) gmres_backsolve_body(a.gdev, a.coef);
}
// flags[i] = member i continues its Arnoldi steps
__global__ void k_ls_cont(const LsMember *t, int count, int *flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) flags[i] = t[i].live && t[i].gdev->cont ? 1 : 0;
}
// One CTA: the step's conditional-node handle = whether any member continues (the replayed cycle).
__global__ void __launch_bounds__(1024) k_ls_cont_cond(const LsMember *t, int count, cudaGraphConditionalHandle h) {
    int any = 0;
    for (int i = threadIdx.x; i < count; i += blockDim.x) any |= t[i].live && t[i].gdev->cont;
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) cudaGraphSetConditional(h, any ? 1 : 0);
}
// the host-read record of every member's cycle (beta, |r|^2, iterations, basis size, status)
struct LsTail {
    double beta, rnorm2;
    int iters, count, status, pad;
};
__global__ void k_ls_tails(const LsMember *t, int count, LsTail *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const GmresDev *d = t[i].gdev;
    out[i] = LsTail{d->beta, d->rnorm2, d->iters, d->count, d->status, 0};
}

// ---- block-Jacobi solve z = M^{-1} src over the members [first, first + count) of one layout ----
// The solve bodies keep the compiler's own FMA choices (they pair FP32 operations and are
// faster than any explicitly rounded form); that they compute the same bits here as in
// k_lu_solve / k_lu_solve_half is checked by the lockstep tests, member by member.
template <typename T, bool DIAG>
__global__ void __launch_bounds__(SOLVE_THREADS, (solve_min_blocks<T, DIAG>()))
k_ls_solve(const LsMember *t, int first, int count, int src, int dst, int j, int gate) {
    const int i = ls_find(t, first, count, blockIdx.x, LS_SOLVE);
    const LsMember &a = t[i];
    if (!ls_on(a, gate)) return;
    const int blocks = (i + 1 < first + count ? t[i + 1].solve0 : gridDim.x) - a.solve0;
    lu_solve_body<T, DIAG>(blockIdx.x - a.solve0, blocks, (const T *)a.pool, a.perm, a.stride, a.m, a.cells,
                           ls_vec(a, src, j), ls_vec(a, dst, j));
}
__global__ void __launch_bounds__(SOLVE_THREADS, 5)
k_ls_solve_half(const LsMember *t, int first, int count, int src, int dst, int j, int gate) {
    const int i = ls_find(t, first, count, blockIdx.x, LS_SOLVE);
    const LsMember &a = t[i];
    if (!ls_on(a, gate)) return;
    const int blocks = (i + 1 < first + count ? t[i + 1].solve0 : gridDim.x) - a.solve0;
    lu_solve_half_body(blockIdx.x - a.solve0, blocks, (const __half *)a.pool, a.scale, a.perm, a.m, a.cells,
                       ls_vec(a, src, j), ls_vec(a, dst, j));
}

// ---- face-block Jacobi of HDG members from FP32 inverses (k_inv_apply's body) ----------------
__global__ void __launch_bounds__(INV_APPLY_THREADS)
k_ls_inv_apply(const LsMember *t, int first, int count, int src, int dst, int j, int gate) {
    const int i = ls_find(t, first, count, blockIdx.x, LS_SOLVE);
    const LsMember &a = t[i];
    if (!ls_on(a, gate)) return;
    const int blocks = (i + 1 < first + count ? t[i + 1].solve0 : gridDim.x) - a.solve0;
    inv_apply_body(blockIdx.x - a.solve0, blocks, (const float *)a.pool, a.m, a.cells, ls_vec(a, src, j),
                   ls_vec(a, dst, j));
}

// ---- condensed Schur apply of HDG members [first, first + count), all of degree N - 1 ----------
template <int N>
__global__ void __launch_bounds__(256) k_ls_hdg_apply(const LsMember *t, int first, int count, int src, int dst,
                                                      int gate) {
    const LsMember &a = t[ls_find(t, first, count, blockIdx.x, LS_TEAM)];
    if (!ls_on(a, gate)) return;
    const int face = blockIdx.x - a.team0;
    if (a.c32) hdg_apply32_body<N>(face, (const float *)a.S, a.speeds, ls_vec(a, src, 0), ls_vec(a, dst, 0), *a.basis, a.g);
    else hdg_apply_body<N>(face, (const double *)a.S, a.speeds, ls_vec(a, src, 0), ls_vec(a, dst, 0), *a.basis, a.g);
}

// ---- J·v of the members [first, first + count), all of degree N - 1 --------------------------
template <int N>
__global__ void __launch_bounds__(Team<N>::THREADS) k_ls_face_trace(const LsMember *t, int first, int count, int src,
                                                                    int gate) {
    const LsMember &a = t[ls_find(t, first, count, blockIdx.x, LS_TEAM)];
    if (!ls_on(a, gate)) return;
    face_trace_body<N, false>(blockIdx.x - a.team0, ls_vec(a, src, 0), a.traces, *a.basis, a.g, nullptr);
}
template <int N>
__global__ void __launch_bounds__(Team<N>::THREADS, 65536 / (Team<N>::THREADS * 72))
k_ls_dg_apply(const LsMember *t, int first, int count, int src, int dst, int gate) {
    const LsMember &a = t[ls_find(t, first, count, blockIdx.x, LS_TEAM)];
    if (!ls_on(a, gate)) return;
    dg_apply_body<N>(blockIdx.x - a.team0, ls_vec(a, src, 0), a.traces, a.vol, a.fcache, a.speeds, ls_vec(a, dst, 0),
                     a.basis, a.g, a.inv_step, 1);
}

}  // namespace dgh
