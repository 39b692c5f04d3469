// C ABI of the B200 DG / condensed-HDG Euler solver: context, memory pools, kernel launches,
// the block-Jacobi preconditioners and the device-resident GMRES(m).  A context solves either
// the 2D problem (dg_hdg_2d) or, with dgh_config.dim = 1, the 1D problem (dg_hdg_1d); the two
// share the GMRES, the Arnoldi kernels, the vector helpers and the host integrator, and differ
// in their discretisation kernels (dgh_kernels_dg/hdg.cuh versus dgh_kernels_1d.cuh).
#include "dgh_gpu.h"
#include "host/slab.hpp"
#include "dgh_kernels_1d.cuh"
#include "dgh_kernels_ilu1d.cuh"
#include "dgh_kernels_ilu2d.cuh"
#include "dgh_kernels_dg.cuh"
#include "dgh_kernels_hdg.cuh"
#include "dgh_kernels_init.cuh"
#include "dgh_kernels_krylov.cuh"
#include "dgh_kernels_lu.cuh"
#include "dgh_kernels_lu2.cuh"
#include "dgh_kernels_lockstep.cuh"
#include "dgh_kernels_q.cuh"

#include <cublas_v2.h>

#include <algorithm>
#include <condition_variable>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <stdexcept>
#include <tuple>
#include <string>
#include <vector>

using namespace dgh;

namespace {
struct Failure {
    int code;
    std::string message;
};
[[noreturn]] void fail(int code, const std::string &m) { throw Failure{code, m}; }
void ck(cudaError_t e, const char *what) {
    if (e != cudaSuccess) fail(DGH_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Gauss-Legendre rule by Newton's method on P_n in extended precision (ascending nodes).
void gauss_rule(int n, std::vector<double> &x, std::vector<double> &w) {
    x.assign(n, 0.);
    w.assign(n, 0.);
    const double pi = std::acos(-1.);
    for (int k = 0; k < (n + 1) / 2; ++k) {
        long double z = std::cos(pi * (k + .75) / (n + .5)), p0 = 1, p1 = z, dp = 1;
        auto eval = [&]() {
            p0 = 1;
            p1 = z;
            for (int j = 2; j <= n; ++j) {
                long double p2 = ((2 * j - 1) * z * p1 - (j - 1) * p0) / j;
                p0 = p1;
                p1 = p2;
            }
            if (n == 1) { p1 = z; p0 = 1; }
            dp = n * (z * p1 - p0) / (z * z - 1);
        };
        for (int it = 0; it < 100; ++it) {
            eval();
            long double dz = p1 / dp;
            z -= dz;
            if (std::fabs((double)dz) <= 1e-19) break;
        }
        eval();
        x[n - 1 - k] = (double)z;
        x[k] = -(double)z;
        w[k] = w[n - 1 - k] = (double)(2 / ((1 - z * z) * dp * dp));
    }
    if (n % 2) x[n / 2] = 0;
}
std::vector<double> lagrange(const std::vector<double> &x, double z) {
    const int n = (int)x.size();
    std::vector<double> v(n, 1.);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            if (i != j) v[i] *= (z - x[j]) / (x[i] - x[j]);
    return v;
}
constexpr int RED_BLOCKS_PER_SM = 4;
}  // namespace

struct dgh_ctx {
    dgh_config cfg{};
    int dim = 2, Q = 0;  // Q: quadrature points per direction (1D may over-integrate)
    int n = 0, P = 0, m = 0, cells = 0, faces = 0, fw = 0, t = 0, restart = 0;
    size_t nspeeds = 0;  // doubles of the frozen speeds: 2 per face node (2D) or per face (1D)
    Basis1Q b1{};        // 1D reference element with its quadrature rule
    Grid1 g1{};
    long long N = 0, NT = 0;
    Grid g{};
    Basis1D basis{};
    Basis1D *basis_dev = nullptr;  // device copy, for tables indexed per thread
    BasisQ *bq = nullptr;          // 2D over-integration: the volume rule (Q > n)
    double *volq = nullptr;        // (u, v, H) at the volume points [cell][Q*Q][3]
    Case cs{};
    double step_size = 0, inv_step = 0;
    int sms = 148, red_grid = 592;
    cudaStream_t stream = nullptr;
    std::string err;
    int64_t launches = 0;
    size_t bytes = 0;
    std::vector<void *> owned;
    std::vector<double> xnodes;
    // device buffers
    ErrorRule *rule = nullptr;
    double *old = nullptr, *inv_mass = nullptr, *mass = nullptr, *inv_trace_mass = nullptr;
    double *speeds = nullptr, *traces = nullptr, *traces2 = nullptr, *partial = nullptr, *red = nullptr;
    double *vol = nullptr, *fcache = nullptr;
    int *status = nullptr, *ok = nullptr;
    double *pinned = nullptr;  // host pinned scratch for scalar read-back
    bool frozen = false, linearised = false, dg_factored = false, condensed = false, face_factored = false;
    // DG block Jacobi pool (precision per cfg.precision)
    void *dg_pool = nullptr;
    int *dg_perm = nullptr;
    // HDG condensation
    double *S = nullptr, *X = nullptr, *Y = nullptr, *cy = nullptr, *hrhs = nullptr;
    double *aug = nullptr;
    int *aug_perm = nullptr;
    int aug_cells = 0;
    size_t aug_bytes = 0;
    void *face_pool = nullptr;
    int *face_perm = nullptr;
    bool face_inverse = false;  // mixed 2D: face_pool holds FP32 explicit inverses
    // FP32 condensation (dgh_config.condense32, 2D): the cells' LU factors of A in FP32 slabs
    // with their permutations, the Schur blocks in FP32, the FP32 view of the condensation
    // workspace, and a volume scratch vector for the recovery
    float *S32 = nullptr, *lu32 = nullptr, *aug32 = nullptr;
    int *lu32_perm = nullptr;
    double *hq = nullptr;
    bool c32() const { return cfg.condense32 != 0 && dim == 2; }
    // 1D block ILU(0): the periodic block pattern, its symbolic update schedule, the pattern
    // blocks (row-major, slot order) and the diagonal blocks' permutations, per operator
    struct IluPlan {
        int rows = 0, m = 0, nnz = 0;
        int *row_ptr = nullptr, *col = nullptr, *diag = nullptr, *slot_row = nullptr;
        int *upd_off = nullptr, *upd_target = nullptr, *upd_upper = nullptr, *perm = nullptr;
        void *vals = nullptr;
    } ilu_dg, ilu_hdg;
    // 2D block ILU(0) of the DG operator on the periodic cartesian block graph, natural ordering:
    // per row (cell) the diagonal block and the 4 neighbour blocks in increasing column order
    // (the lower ones first); forward and backward level schedules; per forward level and lower
    // slot order q the batched products of the factorisation (pointer arrays on the device)
    struct Ilu2 {
        bool on = false;
        void *diag = nullptr, *offd = nullptr;  // factor storage (FP64, or FP32 in the mixed forms)
        int *nlower = nullptr, *ncol = nullptr, *frows = nullptr, *brows = nullptr, *pairs = nullptr;
        void **cdst = nullptr;                  // coupling block of pair k
        std::vector<int> fptr, bptr;            // level offsets into frows / brows
        struct Batch {
            int n = 0;
            void **a = nullptr, **b = nullptr, **c = nullptr;
        };
        struct Step {
            Batch mult, update;
        };
        std::vector<std::array<Step, 4>> steps;
        void *scratch = nullptr;
        double *aug = nullptr, *inv = nullptr, *ydummy = nullptr, *work = nullptr, *tvec = nullptr;
        int *perm = nullptr;
        cublasHandle_t blas = nullptr;
    } ilu2;
    bool ilu2d() const { return ilu() && dim == 2; }
    bool ilu() const { return cfg.preconditioner == 1; }
    // left-looking FP64 LU: per-CTA scratch of the panels' L_qq^{-1}, U_qq^{-1}; FP64 workspace
    // for the mixed-precision DG blocks (factored in FP64 in chunks, stored as FP32 slabs)
    double *lu_tri = nullptr, *dg_ws = nullptr;
    int lu_grid = 0, dg_ws_cells = 0;
    // per-degree autotuner: chosen factorisation variants (-1 until the first refresh) and the
    // tuning times
    int dg_variant = -1, hdg_variant = -1;
    double tune_ms[4] = {0, 0, 0, 0};
    // grid shape of the DG block solves (solve_grid; -1 until the first DG refresh) and its tuning times
    int solve_shape = -1;
    double solve_ms[2] = {0, 0};
    // CTAs per SM of the fused DG factorisation (1 or 2; -1 until the first fused refresh): with
    // 1 the per-CTA FP64 slots fit L2, with 2 twice the warps hide the panel latencies
    int fused_ctas = -1;
    double fused_ms[2] = {0, 0};
    // GMRES
    double *V = nullptr, *gw = nullptr, *gz = nullptr, *gres[3] = {nullptr, nullptr, nullptr}, *gcoef = nullptr;
    double *g_rhs = nullptr, *g_x = nullptr;  // the solve's own copies of rhs and x (fixed graph operands)
    GmresDev *gdev = nullptr;
    long long vld = 0;
    // lockstep batch this context's DG GMRES solves join while a session is open (-1: none)
    dgh_lockstep *ls = nullptr;
    int ls_index = -1;
    // slab of a decomposed mesh (dgh_ctx_create_slab): global rows [row0, row0 + rows) of ny,
    // held as local rows 1..rows above ghost row 0 and below `above` ghost rows (1 for the DG
    // operator; 2 for HDG, whose top ghost cells are condensed and need their own upper faces);
    // row_len doubles per cell row of a volume vector, face_row per face row of a trace vector;
    // the halo plans of volume and trace vectors; buf: device scratch of host collectives
    struct Slab {
        dgh_comm *comm = nullptr;
        int row0 = 0, rows = 0, ny = 0, above = 1;
        long long row_len = 0, face_row = 0;
        dgh_halo_plan vol, trace;
        double *buf = nullptr;
    } slab;
    bool slabbed() const { return slab.comm != nullptr; }
    // a host value reduced over the slab ranks (op 0 sum, 1 maximum); the value itself otherwise
    void slab_reduce(double *v, int count, int op) {
        if (!slabbed()) return;
        ck(cudaMemcpyAsync(slab.buf, v, count * sizeof(double), cudaMemcpyHostToDevice, stream), "copy");
        slab.comm->allreduce(slab.buf, count, op, stream);
        ck(cudaMemcpyAsync(pinned + 8, slab.buf, count * sizeof(double), cudaMemcpyDeviceToHost, stream), "copy");
        sync();
        std::memcpy(v, pinned + 8, count * sizeof(double));
    }
    // one captured restart cycle per operator (conditional Arnoldi steps), rebuilt when the
    // captured stage scalar (1/tau, a kernel argument of J*v) changes
    struct CycleGraph {
        cudaGraphExec_t exec = nullptr;
        double inv_step = 0;
        int launches_fixed = 0, launches_step = 0;
    } cycle[3];
    bool use_graph = false;
    cudaStream_t aux = nullptr;  // captures the conditional bodies
    // optional CUDA-event timers per kernel class (dgh_timing_enable / dgh_timing_read)
    struct TimerRec { int cat; cudaEvent_t a, b; };
    bool timing = false;
    std::vector<TimerRec> pending;
    std::vector<cudaEvent_t> spare;
    double t_ms[DGH_TIMER_COUNT] = {};
    int64_t t_n[DGH_TIMER_COUNT] = {};
    cudaEvent_t event() {
        if (spare.empty()) {
            cudaEvent_t e;
            ck(cudaEventCreate(&e), "cudaEventCreate");
            return e;
        }
        cudaEvent_t e = spare.back();
        spare.pop_back();
        return e;
    }
    void flush_timers() {
        if (pending.empty()) return;
        ck(cudaStreamSynchronize(stream), "sync");
        for (auto &r : pending) {
            float ms = 0;
            ck(cudaEventElapsedTime(&ms, r.a, r.b), "cudaEventElapsedTime");
            t_ms[r.cat] += ms;
            t_n[r.cat] += 1;
            spare.push_back(r.a);
            spare.push_back(r.b);
        }
        pending.clear();
    }

    template <class T> T *alloc(size_t count) {
        void *p = nullptr;
        const size_t b = std::max<size_t>(count * sizeof(T), 16);
        ck(cudaMalloc(&p, b), "cudaMalloc");
        owned.push_back(p);
        bytes += b;
        return static_cast<T *>(p);
    }
    void launched(int k = 1) {
        launches += k;
        ck(cudaGetLastError(), "kernel launch");
    }
    // A slab context waits through its communicator (an NCCL rank gives up on a peer that never
    // joins a collective instead of blocking for good).
    void sync();
    bool mixed() const { return cfg.precision != DGH_PRECISION_FP64; }
    bool half16() const { return cfg.precision == DGH_PRECISION_MIXED16; }
    float *dg_scale = nullptr;  // FP16 DG factors: per-row reciprocal scales of U
    double *dg_slots = nullptr; // reduced-precision DG factorisation: one FP64 slot per resident LU CTA
    int dg_slot_count = 0;
    bool d1() const { return dim == 1; }
    bool overint() const { return dim == 2 && Q > n; }
    bool has_dg() const { return cfg.method == DGH_METHOD_DG || cfg.method == DGH_METHOD_BOTH; }
    bool has_hdg() const { return cfg.method == DGH_METHOD_HDG || cfg.method == DGH_METHOD_BOTH; }
    int team_blocks(int cpb) const { return (cells + cpb - 1) / cpb; }
    // Deterministic weighted reduction helpers (return host values).
    // interior: x is a volume vector whose ghost rows a slab must skip (otherwise its ghost rows
    // or faces are zero)
    double reduce_scalar(const double *x, const double *W, bool divide, long long n_, bool interior = false) {
        if (slabbed() && interior) {  // the interior rows, summed over the ranks
            x += slab.row_len;
            W += slab.row_len;
            n_ = (long long)slab.rows * slab.row_len;
        }
        k_wnorm2<<<red_grid, KR_THREADS, 0, stream>>>(x, W, divide ? 1 : 0, n_, partial);
        k_reduce<<<1, KR_THREADS, 0, stream>>>(partial, red_grid, red);
        launched(2);
        if (slabbed()) slab.comm->allreduce(red, 1, 0, stream);
        ck(cudaMemcpyAsync(pinned, red, sizeof(double), cudaMemcpyDeviceToHost, stream), "copy");
        sync();
        return pinned[0];
    }
    void check_status(int mask_clear = 0) {
        int s = 0;
        ck(cudaMemcpyAsync(pinned, status, sizeof(int), cudaMemcpyDeviceToHost, stream), "copy status");
        sync();
        std::memcpy(&s, pinned, sizeof(int));
        if (slabbed()) {  // every rank raises the union of the ranks' status bits
            double bits[8];
            for (int i = 0; i < 8; ++i) bits[i] = (s >> i) & 1;
            slab_reduce(bits, 8, 1);
            for (int i = 0; i < 8; ++i) s |= bits[i] > 0 ? 1 << i : 0;
        }
        if (s) {
            ck(cudaMemsetAsync(status, 0, sizeof(int), stream), "memset");
            (void)mask_clear;
            if (s & ST_FROZEN_FACE) fail(DGH_ERR_STATE, "Invalid frozen face state");
            if (s & ST_CFL_VOLUME) fail(DGH_ERR_STATE, "Invalid CFL volume state");
            if (s & ST_NONPHYS_MEAN) fail(DGH_ERR_STATE, "Nonphysical cell average");
            if (s & ST_SHOCK) fail(DGH_ERR_STATE, "Simple wave reaches shock time");
            if (s & ST_SINGULAR) fail(DGH_ERR_SINGULAR, "Singular block Jacobi factor");
            if (s & ST_SINGULAR_HDG) fail(DGH_ERR_SINGULAR, "Singular or nonfinite LU factors");
            if (s & ST_LU_INPUT) fail(DGH_ERR_SINGULAR, "Nonfinite block LU input");
            fail(DGH_ERR_CUDA, "unknown device status");
        }
    }
};

// A lockstep group of DG GMRES solves (dgh_kernels_lockstep.cuh): the member contexts in table
// order (sorted by degree, so every degree and every factor layout is one contiguous range of
// the table), the launch plan, and the rendezvous of a session, in which each expected member
// brings one DG GMRES solve.  The member that completes the count issues the whole lockstep
// solve on the group's stream; the others wait, then continue on their own streams.
struct dgh_lockstep {
    int device = 0, restart = 0, precision = 0, op = DGH_OP_DG;
    cudaStream_t stream = nullptr;
    cudaEvent_t finished = nullptr;
    std::vector<dgh_ctx *> members;
    struct Range {
        int first = 0, count = 0, key = 0, blocks = 0;
        size_t smem = 0;
    };
    std::vector<Range> degrees;  // operator launches (J·v or Schur apply): key = n (nodes per direction)
    // block-Jacobi launches: key 0 FP64 LU, 1 FP32 LU, 2 FP32 LU narrow (m < 64), 3 FP16 LU,
    // 4 FP32 inverses (HDG face blocks); for HDG groups re-planned every session
    std::vector<Range> layouts;
    std::vector<int> layout_keys;  // the keys the captured cycle graph was built with
    int red_total = 0;
    LsMember *table = nullptr, *host = nullptr;  // device table and its pinned host image
    int *flags = nullptr, *flags_host = nullptr;
    LsTail *tails = nullptr, *tails_host = nullptr;
    struct Slot {
        bool arrived = false, withdrawn = false, trivial = false;
        double tol = 0, rhs_norm = 0, rel = 0;
        int limit = 0, iters = 0, code = DGH_OK;
        std::string msg;
        cudaEvent_t ready = nullptr;
    };
    std::vector<Slot> slots;
    std::mutex mu;
    std::condition_variable cv;
    bool open = false;
    int expected = 0, arrived = 0, withdrawn = 0;
    uint64_t generation = 0;
    int64_t sessions = 0, cycles = 0, steps = 0, launches = 0;
    // the restart cycle captured once as a CUDA graph (used when every member replays its own
    // cycles as graphs): the kernels read the member table, so one graph serves every session
    cudaGraphExec_t cycle = nullptr;
    cudaStream_t aux = nullptr;
    int graph_fixed = 0, graph_step = 0;
    void launched(int k = 1) {
        launches += k;
        ck(cudaGetLastError(), "kernel launch");
    }
};

void dgh_ctx::sync() {
    if (slab.comm) slab.comm->wait(stream);
    else ck(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
}

namespace {
// A slab context whose call fails on its own (a CUDA or communication error, which its peers
// cannot have seen) fails its communicator, so that the peer ranks leave their next collective
// with DGH_ERR_COMM instead of waiting for it.  Failures decided from reduced values (norms,
// status bits, GMRES counts) happen on every rank alike and leave the group usable.
template <class F> int guard(dgh_ctx *ctx, F &&f) {
    if (!ctx) return DGH_ERR_INVALID;
    int code = DGH_OK;
    try {
        f();
        return DGH_OK;
    } catch (const Failure &e) {
        ctx->err = e.message;
        code = e.code;
    } catch (const dgh_comm_failure &e) {
        ctx->err = e.what();
        code = DGH_ERR_COMM;
    } catch (const std::exception &e) {
        ctx->err = e.what();
        code = DGH_ERR_CUDA;
    }
    if (ctx->slabbed() && (code == DGH_ERR_CUDA || code == DGH_ERR_COMM)) ctx->slab.comm->fail(ctx->err);
    return code;
}
void need(bool c, const char *m) {
    if (!c) fail(DGH_ERR_INVALID, m);
}
// Records an event pair around a region when timing is enabled.
struct Timed {
    dgh_ctx *c;
    int cat;
    cudaEvent_t a = nullptr;
    Timed(dgh_ctx *ctx, int category) : c(ctx), cat(category) {
        if (c->timing) {
            a = c->event();
            ck(cudaEventRecord(a, c->stream), "cudaEventRecord");
        }
    }
    ~Timed() {
        if (a) {
            cudaEvent_t b = c->event();
            cudaEventRecord(b, c->stream);
            c->pending.push_back({cat, a, b});
            if (c->pending.size() > 2048) c->flush_timers();
        }
    }
};

#define DGH_DISPATCH_N(nn, ...)               \
    switch (nn) {                             \
        case 1: { constexpr int N = 1; __VA_ARGS__; } break; \
        case 2: { constexpr int N = 2; __VA_ARGS__; } break; \
        case 3: { constexpr int N = 3; __VA_ARGS__; } break; \
        case 4: { constexpr int N = 4; __VA_ARGS__; } break; \
        case 5: { constexpr int N = 5; __VA_ARGS__; } break; \
        case 6: { constexpr int N = 6; __VA_ARGS__; } break; \
        case 7: { constexpr int N = 7; __VA_ARGS__; } break; \
        case 8: { constexpr int N = 8; __VA_ARGS__; } break; \
        case 9: { constexpr int N = 9; __VA_ARGS__; } break; \
        default: fail(DGH_ERR_INVALID, "Unsupported face degree"); \
    }

// ---- launch helpers ---------------------------------------------------------------------------
constexpr int K1_THREADS = 128;
inline unsigned grid1(long long n, int t = K1_THREADS) { return (unsigned)((n + t - 1) / t); }
void launch_trace(dgh_ctx *c, const double *u, double *tr, bool check) {
    if (c->d1()) {
        DGH_DISPATCH_N(c->n, {
            if (check) k1_traces<N, true><<<grid1(c->cells), K1_THREADS, 0, c->stream>>>(u, tr, c->b1, c->g1, c->ok);
            else k1_traces<N, false><<<grid1(c->cells), K1_THREADS, 0, c->stream>>>(u, tr, c->b1, c->g1, c->ok);
        });
        c->launched();
        return;
    }
    DGH_DISPATCH_N(c->n, {
        using T = Team<N>;
        if (check) k_face_trace<N, true><<<c->team_blocks(T::CPB), T::THREADS, 0, c->stream>>>(u, tr, c->basis, c->g, c->ok);
        else k_face_trace<N, false><<<c->team_blocks(T::CPB), T::THREADS, 0, c->stream>>>(u, tr, c->basis, c->g, c->ok);
        if (check && c->overint()) {  // the over-integrated rule also checks its volume points
            k_points_check_q<N><<<std::min(c->cells, c->sms * 4), Q_THREADS, 0, c->stream>>>(u, c->bq, c->g, c->ok);
            c->launched();
        }
    });
    c->launched();
}

// Slab contexts: the ghost rows of a volume vector filled from the neighbouring slabs (before a
// kernel reads neighbour cells), or cleared (outputs whose ghost rows hold no equation).  The
// library owns the ghost rows of the vectors passed to it, const or not.
void slab_halo(dgh_ctx *c, const double *v) {
    if (c->slabbed()) c->slab.comm->exchange(const_cast<double *>(v), c->slab.vol, c->stream);
}
void slab_zero_ghosts(dgh_ctx *c, double *v) {
    if (!c->slabbed()) return;
    const size_t row = (size_t)c->slab.row_len;
    ck(cudaMemsetAsync(v, 0, row * sizeof(double), c->stream), "memset");
    ck(cudaMemsetAsync(v + (c->slab.rows + 1) * row, 0, c->slab.above * row * sizeof(double), c->stream), "memset");
}
// Trace vectors of a slab (HDG): the owned faces are the x faces and the upper y faces of the
// slab's own rows.  The halo brings the faces the Schur apply, the recovery and the recovered
// residual of owned faces and interior cells read: the lower y faces of row 1 (owned by the rank
// below), and the x and upper y faces of the first ghost row above (owned by the rank above).
void slab_trace_halo(dgh_ctx *c, const double *v) {
    if (c->slabbed()) c->slab.comm->exchange(const_cast<double *>(v), c->slab.trace, c->stream);
}
void slab_zero_ghost_faces(dgh_ctx *c, double *v) {
    if (!c->slabbed()) return;
    const size_t fr = (size_t)c->slab.face_row, y0 = (size_t)c->cells * c->fw;
    const size_t top = (size_t)(c->slab.rows + 1) * fr, tail = (size_t)c->slab.above * fr;
    for (size_t base : {(size_t)0, y0}) {
        ck(cudaMemsetAsync(v + base, 0, fr * sizeof(double), c->stream), "memset");
        ck(cudaMemsetAsync(v + base + top, 0, tail * sizeof(double), c->stream), "memset");
    }
}
// Device values summed over the slab ranks in place (the Arnoldi coefficients and norms).
void slab_sum(dgh_ctx *c, double *dev, int count) {
    if (c->slabbed()) c->slab.comm->allreduce(dev, count, 0, c->stream);
}
// The interior cells of a slab (all cells otherwise): [first, first + count).
void interior_cells(const dgh_ctx *c, int &first, int &count) {
    first = c->slabbed() ? c->g.nx : 0;
    count = c->slabbed() ? c->g.nx * c->slab.rows : c->cells;
}

// The dynamic shared-memory cap of a kernel is process-wide state that every context shares (and
// the contexts of a batch run on several host threads): it only ever rises, under a lock, so no
// launch sees a cap below the size it was launched with.
void allow_dynamic_smem(const void *fn, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, size_t> cap;
    int dev = 0;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lock(mu);
    size_t &cur = cap[{fn, dev}];
    if (bytes <= cur) return;
    ck(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes), "shared memory attribute");
    cur = bytes;
}

// Panel width 32; U12 tile width 32 for FP64 (two CTAs per SM fit in shared memory at m = 324)
// and 64 for FP32.
constexpr int LU_NB = 32;
template <typename TF> constexpr int lu_tc() { return sizeof(TF) == 8 ? 32 : 64; }
template <typename TF> void setup_lu_attrs(size_t smem) {
    allow_dynamic_smem((const void *)k_lu<TF, LU_NB, lu_tc<TF>()>, smem);
}
template <typename TF>
void launch_lu(dgh_ctx *c, TF *pool, size_t stride, int m, int ld, int count, int *perm, int bit, bool slab_out,
               bool lfix = false) {
    constexpr int TC = lu_tc<TF>();
    const size_t smem = lu_smem_bytes<TF, LU_NB, TC>(m);
    setup_lu_attrs<TF>(smem);
    int per_sm = 0;
    ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lu<TF, LU_NB, TC>, LU_THREADS, smem), "occupancy");
    const int grid = std::min(count, c->sms * std::max(1, per_sm));
    k_lu<TF, LU_NB, TC><<<grid, LU_THREADS, smem, c->stream>>>(pool, stride, m, ld, count, perm, c->status, bit,
                                                               slab_out ? 3 : lfix ? 2 : 0);
    c->launched();
}
// The left-looking FP64 LU (dgh_kernels_lu2.cuh): grid = resident CTAs, each with its scratch.
template <bool AUG>
void launch_lu_left(dgh_ctx *c, double *pool, size_t stride, int m, int ld, int count, int *perm, int bit, bool slab_out,
                    float *out32 = nullptr, double *x_out = nullptr, double *y_out = nullptr) {
    need(m <= 2 * LL_THREADS && m % 4 == 0, "LU block width unsupported by the left-looking kernel");
    const size_t smem = lu_left_smem_bytes(m);
    allow_dynamic_smem((const void *)k_lu_left<AUG>, smem);
    const int grid = std::min(count, c->lu_grid);
    k_lu_left<AUG><<<grid, LL_THREADS, smem, c->stream>>>(pool, stride, m, ld, count, c->lu_tri, perm, c->status, bit,
                                                          slab_out ? 1 : 0, out32, x_out, y_out);
    c->launched();
}
// The DG blocks of cells [first, first + count) assembled and factored in one persistent launch
// (k_lu_left's fused mode: each CTA assembles a cell into its own FP64 slot, factors it there and
// writes FP32 slabs, or FP16 slabs with row scales).  Collocated volume rule only.
template <int N> void launch_dg_fused(dgh_ctx *c, int first, int count) {
    const size_t smem = lu_left_smem_bytes(c->m);
    allow_dynamic_smem((const void *)k_lu_left<false, N>, smem);
    int per_sm = 0;
    ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lu_left<false, N>, LL_THREADS, smem), "occupancy");
    const int per = std::min(std::max(1, per_sm), c->fused_ctas > 0 ? c->fused_ctas : 2);
    const int grid = std::min(count, std::min(c->dg_slot_count, c->sms * per));
    need(grid <= c->lu_grid, "fused factorisation grid exceeds the LU scratch");
    LLFuse fu;
    fu.vol = c->vol;
    fu.fcache = c->fcache;
    fu.speeds = c->speeds;
    fu.slots = c->dg_slots;
    fu.b = c->basis;
    fu.g = c->g;
    fu.inv_step = c->inv_step;
    fu.first = first;
    const size_t mp8 = pad8(c->m);
    float *out32 = nullptr;
    if (c->half16()) {
        fu.out16 = (__half *)c->dg_pool + (size_t)first * c->m * mp8;
        fu.scale16 = c->dg_scale + (size_t)first * c->m;
    } else {
        out32 = (float *)c->dg_pool + (size_t)first * c->m * c->m;
    }
    k_lu_left<false, N><<<grid, LL_THREADS, smem, c->stream>>>(c->dg_slots, (size_t)c->m * c->m, c->m, c->m, count,
                                                                c->lu_tri, c->dg_perm + (size_t)first * c->m, c->status,
                                                                ST_SINGULAR, 0, out32, nullptr, nullptr, fu);
    c->launched();
}

// Narrow blocks (m <= 64): one warp per block in shared memory.
template <typename TF>
void launch_lu_narrow(dgh_ctx *c, TF *pool, int m, int count, int *perm, int bit) {
    need(m <= 64 && m % 4 == 0, "block width unsupported by the narrow LU");
    const size_t smem = lu_narrow_smem_bytes<TF>(m);
    allow_dynamic_smem((const void *)k_lu_narrow<TF>, smem);
    int resident = 0;
    ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, k_lu_narrow<TF>, NARROW_THREADS, smem), "occupancy");
    constexpr int wpc = NARROW_THREADS / 32;
    const int grid = std::min((count + wpc - 1) / wpc, c->sms * std::max(1, resident));
    k_lu_narrow<TF><<<grid, NARROW_THREADS, smem, c->stream>>>(pool, m, count, perm, c->status, bit);
    c->launched();
}
// Grid of a one-warp-per-block solve over `count` blocks with `wpc` warps per CTA and `resident`
// CTAs per SM.  Shape 0 fills every resident CTA slot, so the last round of blocks runs on the
// few warps whose share is one block larger; shape 1 takes the fewest CTAs that keep the same
// number of rounds, so every warp solves the same number of blocks (a few one less) with fewer
// warps in flight.  Which is faster depends on the degree and the block count (the autotuner's
// solve-shape kind).
int solve_grid(const dgh_ctx *c, long long count, int wpc, int resident, int shape) {
    const long long want = (count + wpc - 1) / wpc;
    const long long full = std::min<long long>(want, (long long)c->sms * std::max(1, resident));
    if (shape != 1 || full <= 0) return (int)full;
    const long long rounds = (count + full * wpc - 1) / (full * wpc);
    return (int)((count + wpc * rounds - 1) / (wpc * rounds));
}
// One warp per block; enough warps for every SM to keep its warp slots (and their loads) busy.
// FP32 blocks narrower than two slabs (the HDG face blocks) use the register-held diagonal rows.
template <typename TF, bool DIAG>
void launch_solve_as(dgh_ctx *c, const TF *pool, const int *perm, size_t stride, int m, int count, const double *x,
                     double *z, int shape) {
    constexpr int wpc = SOLVE_THREADS / 32;
    const size_t smem = sizeof(TF) * (size_t)m * wpc;
    int resident = 0;
    ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, k_lu_solve<TF, DIAG>, SOLVE_THREADS, smem), "occupancy");
    const int grid = solve_grid(c, count, wpc, resident, shape);
    k_lu_solve<TF, DIAG><<<grid, SOLVE_THREADS, smem, c->stream>>>(pool, perm, stride, m, count, x, z);
    c->launched();
}
template <typename TF>
void launch_solve(dgh_ctx *c, const TF *pool, const int *perm, size_t stride, int m, int count, const double *x,
                  double *z, int shape = 0) {
    if constexpr (sizeof(TF) == 4)
        if (m < 64) return launch_solve_as<TF, true>(c, pool, perm, stride, m, count, x, z, shape);
    launch_solve_as<TF, false>(c, pool, perm, stride, m, count, x, z, shape);
}

template <typename TF>
void launch_solve_t(dgh_ctx *c, const TF *pool, const int *perm, size_t stride, int m, int count, const double *x,
                    double *z) {
    constexpr int wpc = SOLVE_THREADS / 32;
    const size_t smem = sizeof(TF) * (size_t)m * wpc;
    const int want = (count + wpc - 1) / wpc;
    int resident = 0;
    ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, k_lu_solve_t<TF>, SOLVE_THREADS, smem), "occupancy");
    const int grid = std::min(want, c->sms * std::max(1, resident));
    k_lu_solve_t<TF><<<grid, SOLVE_THREADS, smem, c->stream>>>(pool, perm, stride, m, count, x, z);
    c->launched();
}

// The DG cell blocks from their FP16 slabs (one warp per block, like launch_solve).
void launch_solve_half(dgh_ctx *c, const double *x, double *z, int shape) {
    constexpr int wpc = SOLVE_THREADS / 32;
    const size_t smem = sizeof(float) * (size_t)pad8(c->m) * wpc;
    int resident = 0;
    ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, k_lu_solve_half, SOLVE_THREADS, smem), "occupancy");
    const int grid = solve_grid(c, c->cells, wpc, resident, shape);
    k_lu_solve_half<<<grid, SOLVE_THREADS, smem, c->stream>>>((const __half *)c->dg_pool, c->dg_scale, c->dg_perm, c->m,
                                                               c->cells, x, z);
    c->launched();
}

// 1D blocks (m <= 27 and 3 x 3): one warp per block, four warps per CTA.
template <typename TF>
void launch_small_lu(dgh_ctx *c, TF *pool, size_t stride, int m, int ld, int count, int *perm, bool backsolve) {
    const int grid = std::min((count + 3) / 4, c->sms * 16);
    k1_small_lu<TF><<<grid, 128, 0, c->stream>>>(pool, stride, m, ld, count, perm, c->status, ST_LU_INPUT,
                                                 ST_SINGULAR_HDG, backsolve ? 1 : 0);
    c->launched();
}
template <typename TF>
void launch_small_solve(dgh_ctx *c, const TF *pool, const int *perm, int m, int count, const double *x, double *z,
                        bool transpose) {
    const int grid = std::min((count + 3) / 4, c->sms * 16);
    k1_small_solve<TF><<<grid, 128, 0, c->stream>>>(pool, perm, m, count, x, z, transpose ? 1 : 0);
    c->launched();
}

// ---- 2D block ILU(0) of the DG operator ---------------------------------------------------------
void blas_ck(cublasStatus_t e, const char *what) {
    if (e != CUBLAS_STATUS_SUCCESS) fail(DGH_ERR_CUDA, std::string(what) + ": cuBLAS status " + std::to_string((int)e));
}
// The pattern, level schedules and batched-product pointer arrays (block_ilu.cpp:15-45 on the
// cartesian block graph: every row couples to itself and its four face neighbours).
void ilu2_build(dgh_ctx *c) {
    auto &L = c->ilu2;
    const int E = c->cells, m = c->m;
    const size_t mm = (size_t)m * m, tsz = c->mixed() ? sizeof(float) : sizeof(double);
    std::vector<int> ncol(4 * (size_t)E), nlower(E), lev(E, 0), blev(E, 0);
    for (int i = 0; i < E; ++i) {
        int nb[4];
        for (int sd = 0; sd < 4; ++sd) nb[sd] = neighbor(c->g, i, sd);
        std::sort(nb, nb + 4);
        need(nb[0] != nb[1] && nb[1] != nb[2] && nb[2] != nb[3] && nb[0] != i && nb[3] != i,
             "block ILU(0) needs distinct face neighbours (nx, ny >= 3)");
        int nl = 0;
        for (int k = 0; k < 4; ++k) {
            ncol[4 * (size_t)i + k] = nb[k];
            nl += nb[k] < i;
        }
        nlower[i] = nl;
        for (int k = 0; k < nl; ++k) lev[i] = std::max(lev[i], lev[nb[k]] + 1);
    }
    for (int i = E - 1; i >= 0; --i)
        for (int k = nlower[i]; k < 4; ++k) blev[i] = std::max(blev[i], blev[ncol[4 * (size_t)i + k]] + 1);
    auto by_level = [&](const std::vector<int> &lv, std::vector<int> &ptr) {
        const int nlev = *std::max_element(lv.begin(), lv.end()) + 1;
        ptr.assign(nlev + 1, 0);
        for (int i = 0; i < E; ++i) ++ptr[lv[i] + 1];
        for (int l = 0; l < nlev; ++l) ptr[l + 1] += ptr[l];
        std::vector<int> rows(E), fill(ptr.begin(), ptr.end() - 1);
        for (int i = 0; i < E; ++i) rows[fill[lv[i]]++] = i;  // natural order inside a level
        return rows;
    };
    const std::vector<int> frows = by_level(lev, L.fptr), brows = by_level(blev, L.bptr);
    L.diag = c->alloc<char>((size_t)E * mm * tsz);
    L.offd = c->alloc<char>((size_t)E * 4 * mm * tsz);
    auto diag_at = [&](int i) { return (void *)((char *)L.diag + (size_t)i * mm * tsz); };
    auto offd_at = [&](int i, int k) { return (void *)((char *)L.offd + ((size_t)4 * i + k) * mm * tsz); };
    auto slot_in = [&](int i, int col) {  // position of col among row i's neighbours, -1 = diagonal
        if (col == i) return -1;
        for (int k = 0; k < 4; ++k)
            if (ncol[4 * (size_t)i + k] == col) return k;
        return -2;
    };
    // coupling pairs (cell, side) with their destination blocks
    std::vector<int> pairs;
    std::vector<void *> cdst;
    for (int i = 0; i < E; ++i)
        for (int sd = 0; sd < 4; ++sd) {
            pairs.push_back(i);
            pairs.push_back(sd);
            cdst.push_back(offd_at(i, slot_in(i, neighbor(c->g, i, sd))));
        }
    // batched products per forward level and lower slot order (block_ilu.cpp:48-61)
    const int nlev = (int)L.fptr.size() - 1;
    L.steps.assign(nlev, {});
    std::vector<void *> ptrs;
    struct Pending { int l, q; bool update; size_t off; int n; };
    std::vector<Pending> pend;
    size_t max_mult = 1;
    int max_rows = 1;
    for (int l = 0; l < nlev; ++l) {
        max_rows = std::max(max_rows, L.fptr[l + 1] - L.fptr[l]);
        for (int q = 0; q < 4; ++q) {
            std::vector<void *> a, b, cc, ua, ub, uc;
            int k = 0;
            for (int r = L.fptr[l]; r < L.fptr[l + 1]; ++r) {
                const int i = frows[r];
                if (q >= nlower[i]) continue;
                const int j = ncol[4 * (size_t)i + q];
                a.push_back(offd_at(i, q));
                b.push_back(diag_at(j));
                cc.push_back(reinterpret_cast<void *>((size_t)k++));  // scratch index, resolved below
                for (int u = nlower[j]; u < 4; ++u) {  // the upper blocks of row j
                    const int col = ncol[4 * (size_t)j + u], t = slot_in(i, col);
                    if (t == -2) continue;
                    ua.push_back(offd_at(i, q));
                    ub.push_back(offd_at(j, u));
                    uc.push_back(t == -1 ? diag_at(i) : offd_at(i, t));
                }
            }
            max_mult = std::max(max_mult, (size_t)k);
            auto add = [&](std::vector<void *> &x, std::vector<void *> &y, std::vector<void *> &z, bool upd) {
                if (x.empty()) return;
                pend.push_back({l, q, upd, ptrs.size(), (int)x.size()});
                ptrs.insert(ptrs.end(), x.begin(), x.end());
                ptrs.insert(ptrs.end(), y.begin(), y.end());
                ptrs.insert(ptrs.end(), z.begin(), z.end());
            };
            add(a, b, cc, false);
            add(ua, ub, uc, true);
        }
    }
    L.scratch = c->alloc<char>(max_mult * mm * tsz);
    for (const auto &pd : pend)  // scratch indices of the products -> addresses
        if (!pd.update)
            for (int k = 0; k < pd.n; ++k) {
                void *&slot = ptrs[pd.off + 2 * pd.n + k];
                slot = (char *)L.scratch + (size_t)reinterpret_cast<size_t>(slot) * mm * tsz;
            }
    void **dev = c->alloc<void *>(std::max<size_t>(ptrs.size() + cdst.size(), 1));
    ck(cudaMemcpy(dev, ptrs.data(), ptrs.size() * sizeof(void *), cudaMemcpyHostToDevice), "upload ILU pointers");
    ck(cudaMemcpy(dev + ptrs.size(), cdst.data(), cdst.size() * sizeof(void *), cudaMemcpyHostToDevice),
       "upload ILU pointers");
    L.cdst = dev + ptrs.size();
    for (const auto &pd : pend) {
        auto &bt = pd.update ? L.steps[pd.l][pd.q].update : L.steps[pd.l][pd.q].mult;
        bt.n = pd.n;
        bt.a = dev + pd.off;
        bt.b = dev + pd.off + pd.n;
        bt.c = dev + pd.off + 2 * pd.n;
    }
    auto upload_int = [&](const std::vector<int> &v) {
        int *d = c->alloc<int>(v.size());
        ck(cudaMemcpy(d, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice), "upload ILU pattern");
        return d;
    };
    L.ncol = upload_int(ncol);
    L.nlower = upload_int(nlower);
    L.frows = upload_int(frows);
    L.brows = upload_int(brows);
    L.pairs = upload_int(pairs);
    L.aug = c->alloc<double>((size_t)max_rows * m * (2 * m + 1));
    L.inv = c->alloc<double>((size_t)max_rows * mm);
    L.ydummy = c->alloc<double>((size_t)max_rows * m);
    L.perm = c->alloc<int>((size_t)max_rows * m);
    L.work = c->alloc<double>(c->N);
    L.tvec = c->alloc<double>(c->N);
    blas_ck(cublasCreate(&L.blas), "cublasCreate");
    blas_ck(cublasSetStream(L.blas, c->stream), "cublasSetStream");
    L.on = true;
}
// C = alpha A B + beta C for every triple of the batch (row-major m x m blocks: the column-major
// product C^T = B^T A^T).
template <typename TF> void ilu2_gemm(dgh_ctx *c, const dgh_ctx::Ilu2::Batch &bt, TF alpha, TF beta) {
    const int m = c->m;
    if constexpr (sizeof(TF) == 8)
        blas_ck(cublasDgemmBatched(c->ilu2.blas, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, &alpha, (const double *const *)bt.b, m,
                                   (const double *const *)bt.a, m, &beta, (double *const *)bt.c, m, bt.n),
                "cublasDgemmBatched");
    else
        blas_ck(cublasSgemmBatched(c->ilu2.blas, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, &alpha, (const float *const *)bt.b, m,
                                   (const float *const *)bt.a, m, &beta, (float *const *)bt.c, m, bt.n),
                "cublasSgemmBatched");
    c->launched();
}
// BlockPreconditioner::refresh + factorize (block_ilu.cpp:48-61) level by level: every pattern
// block assembled, then per level and lower slot order L_p = A_p A_jj^{-1} and the updates
// A_it -= L_p A_ju, then the level's diagonal blocks inverted (FP64 pivoted LU).
template <typename TF> void ilu2_factor(dgh_ctx *c) {
    auto &L = c->ilu2;
    const int m = c->m, E = c->cells;
    TF *diag = (TF *)L.diag;
    DGH_DISPATCH_N(c->n, {
        k_dg_assemble<N, TF><<<std::min(E, c->sms * 8), 256, 0, c->stream>>>(diag, c->vol, c->fcache, c->speeds, c->basis,
                                                                            c->g, c->inv_step, 0, E, c->overint() ? 0 : 1);
        if (c->overint()) {
            k_vol_block_q<N, TF><<<std::min(E, c->sms * 4), Q_THREADS, 0, c->stream>>>(diag, m, c->volq, c->bq, c->g, 0, E);
            c->launched();
        }
        k_dg_coupling<N, TF><<<std::min(4 * E, c->sms * 8), 256, 0, c->stream>>>((TF *const *)L.cdst, L.pairs, 4 * E,
                                                                                c->fcache, c->speeds, c->basis, c->g);
    });
    c->launched(2);
    const int nlev = (int)L.fptr.size() - 1;
    for (int l = 0; l < nlev; ++l) {
        for (int q = 0; q < 4; ++q) {
            const auto &st = L.steps[l][q];
            if (st.mult.n) {
                ilu2_gemm<TF>(c, st.mult, TF(1), TF(0));
                k_copy_blocks<TF><<<std::min(st.mult.n, c->sms * 4), 256, 0, c->stream>>>(
                    (TF *const *)st.mult.a, (const TF *const *)st.mult.c, st.mult.n, m * m);
                c->launched();
            }
            if (st.update.n) ilu2_gemm<TF>(c, st.update, TF(-1), TF(1));
        }
        const int cnt = L.fptr[l + 1] - L.fptr[l];
        const int *rows = L.frows + L.fptr[l];
        k_ilu_stage_inverse<TF><<<std::min(cnt, c->sms * 4), 256, 0, c->stream>>>(L.aug, diag, rows, cnt, m);
        c->launched();
        launch_lu_left<true>(c, L.aug, (size_t)m * (2 * m + 1), m, 2 * m + 1, cnt, L.perm, ST_SINGULAR, false, nullptr,
                             L.inv, L.ydummy);
        k_ilu_store_inverse<TF><<<std::min(cnt, c->sms * 4), 256, 0, c->stream>>>(diag, L.inv, rows, cnt, m);
        c->launched();
    }
}
// block_ilu.cpp:62-84: forward sweep with L, backward sweep with U and the diagonal inverses,
// level by level; every level's block rows are split over CTAs of ILU_ROWS output rows.
template <typename TF> void ilu2_apply(dgh_ctx *c, const double *x, double *z) {
    auto &L = c->ilu2;
    const int m = c->m, chunks = (m + ILU_ROWS - 1) / ILU_ROWS;
    const TF *offd = (const TF *)L.offd, *diag = (const TF *)L.diag;
    ck(cudaMemcpyAsync(L.work, x, c->N * sizeof(double), cudaMemcpyDeviceToDevice, c->stream), "copy");
    int launches = 0;
    for (int l = 1; l + 1 < (int)L.fptr.size(); ++l) {  // level 0 rows have no lower neighbours
        const int cnt = L.fptr[l + 1] - L.fptr[l];
        k_ilu2_rows<TF, 0><<<cnt * chunks, 256, sizeof(double) * 4 * m, c->stream>>>(
            L.frows + L.fptr[l], cnt, chunks, L.nlower, L.ncol, offd, diag, L.work, L.tvec, z, m);
        ++launches;
    }
    for (int l = 0; l + 1 < (int)L.bptr.size(); ++l) {
        const int cnt = L.bptr[l + 1] - L.bptr[l];
        const int *rows = L.brows + L.bptr[l];
        k_ilu2_rows<TF, 1><<<cnt * chunks, 256, sizeof(double) * 4 * m, c->stream>>>(rows, cnt, chunks, L.nlower, L.ncol,
                                                                                     offd, diag, L.work, L.tvec, z, m);
        k_ilu2_rows<TF, 2><<<cnt * chunks, 256, sizeof(double) * m, c->stream>>>(rows, cnt, chunks, L.nlower, L.ncol,
                                                                                 offd, diag, L.work, L.tvec, z, m);
        launches += 2;
    }
    c->launched(launches);
}

// The DG cell blocks' block-Jacobi solve z = M^{-1} x with grid shape `shape` (solve_grid).
void dg_block_solve(dgh_ctx *c, int shape, const double *x, double *z) {
    const size_t stride = (size_t)c->m * c->m;
    if (c->half16()) launch_solve_half(c, x, z, shape);
    else if (c->mixed()) launch_solve<float>(c, (const float *)c->dg_pool, c->dg_perm, stride, c->m, c->cells, x, z, shape);
    else launch_solve<double>(c, (const double *)c->dg_pool, c->dg_perm, stride, c->m, c->cells, x, z, shape);
}
void precond_apply(dgh_ctx *c, int op, const double *x, double *z) {
    Timed tm(c, DGH_TIMER_PRECOND);
    if (c->d1()) {
        const bool dg = op != DGH_OP_HDG;
        need(dg ? c->dg_factored : c->face_factored, "Refresh the block-Jacobi preconditioner before applying it");
        if (c->ilu()) {
            need(op != DGH_OP_DG_T, "The transposed block ILU(0) is not built");
            const auto &pl = dg ? c->ilu_dg : c->ilu_hdg;
            if (c->mixed())
                k1_ilu_apply<float><<<1, ILU_THREADS, 0, c->stream>>>((const float *)pl.vals, pl.perm, pl.row_ptr, pl.col,
                                                                    pl.diag, pl.rows, pl.m, x, z);
            else
                k1_ilu_apply<double><<<1, ILU_THREADS, 0, c->stream>>>((const double *)pl.vals, pl.perm, pl.row_ptr,
                                                                     pl.col, pl.diag, pl.rows, pl.m, x, z);
            c->launched();
            return;
        }
        const void *pool = dg ? c->dg_pool : c->face_pool;
        const int *perm = dg ? c->dg_perm : c->face_perm, m = dg ? c->m : c->fw;
        if (c->mixed()) launch_small_solve<float>(c, (const float *)pool, perm, m, c->cells, x, z, op == DGH_OP_DG_T);
        else launch_small_solve<double>(c, (const double *)pool, perm, m, c->cells, x, z, op == DGH_OP_DG_T);
        return;
    }
    if (op == DGH_OP_DG_T) {
        need(c->dg_factored, "Refresh the block-Jacobi preconditioner before applying it");
        const size_t stride = (size_t)c->m * c->m;
        need(!c->half16(), "The transposed solve needs FP64 or FP32 factors");
        need(!c->ilu2d(), "The transposed block ILU(0) is not built");
        if (c->mixed()) launch_solve_t<float>(c, (const float *)c->dg_pool, c->dg_perm, stride, c->m, c->cells, x, z);
        else launch_solve_t<double>(c, (const double *)c->dg_pool, c->dg_perm, stride, c->m, c->cells, x, z);
        return;
    }
    if (op == DGH_OP_DG && c->ilu2d()) {
        need(c->dg_factored, "Refresh the block-Jacobi preconditioner before applying it");
        if (c->mixed()) ilu2_apply<float>(c, x, z);
        else ilu2_apply<double>(c, x, z);
        return;
    }
    if (op == DGH_OP_DG) {
        need(c->dg_factored, "Refresh the block-Jacobi preconditioner before applying it");
        dg_block_solve(c, std::max(0, c->solve_shape), x, z);
    } else {
        need(c->face_factored, "Refresh the block-Jacobi preconditioner before applying it");
        const size_t stride = (size_t)c->fw * c->fw;
        if (c->face_inverse) {
            constexpr int wpc = INV_APPLY_THREADS / 32;
            const int grid = std::min((c->faces + wpc - 1) / wpc, c->sms * 8);
            k_inv_apply<<<grid, INV_APPLY_THREADS, 0, c->stream>>>((const float *)c->face_pool, c->fw, c->faces, x, z);
            c->launched();
        } else if (c->mixed())
            launch_solve<float>(c, (const float *)c->face_pool, c->face_perm, stride, c->fw, c->faces, x, z);
        else launch_solve<double>(c, (const double *)c->face_pool, c->face_perm, stride, c->fw, c->faces, x, z);
    }
}

void dg_apply(dgh_ctx *c, const double *v, double *out) {
    need(c->linearised, "Refresh the volume Jacobian before applying it");
    if (c->d1()) {
        DGH_DISPATCH_N(c->n, {
            k1_dg_apply<N><<<grid1(c->cells), K1_THREADS, 0, c->stream>>>(v, c->vol, c->fcache, out, c->b1, c->g1,
                                                                          c->inv_step);
        });
        c->launched();
        return;
    }
    slab_halo(c, v);
    launch_trace(c, v, c->traces2, false);
    DGH_DISPATCH_N(c->n, {
        using T = Team<N>;
        k_dg_apply<N><<<c->team_blocks(T::CPB), T::THREADS, 0, c->stream>>>(v, c->traces2, c->vol, c->fcache, c->speeds,
                                                                            out, c->basis_dev, c->g, c->inv_step,
                                                                            c->overint() ? 0 : 1);
        if (c->overint()) {
            k_vol_apply_q<N><<<std::min(c->cells, c->sms * 4), Q_THREADS, 0, c->stream>>>(v, c->volq, out, c->bq, c->g);
            c->launched();
        }
    });
    c->launched();
    slab_zero_ghosts(c, out);
}
void dg_apply_t(dgh_ctx *c, const double *w, double *out) {
    need(!c->d1(), "The adjoint J^T w is built for the 2D operator only");
    need(!c->slabbed(), "J^T w is not built for slab contexts");
    need(c->linearised, "Refresh the volume Jacobian before applying it");
    launch_trace(c, w, c->traces2, false);
    DGH_DISPATCH_N(c->n, {
        using T = Team<N>;
        k_dg_apply_t<N><<<c->team_blocks(T::CPB), T::THREADS, 0, c->stream>>>(w, c->traces2, c->vol, c->fcache,
                                                                              c->speeds, out, c->basis, c->g,
                                                                              c->inv_step, c->overint() ? 0 : 1);
        if (c->overint()) {
            k_vol_apply_q_t<N><<<std::min(c->cells, c->sms * 4), Q_THREADS, 0, c->stream>>>(w, c->volq, out, c->bq,
                                                                                            c->g);
            c->launched();
        }
    });
    c->launched();
}
void hdg_apply(dgh_ctx *c, const double *lam, double *out) {
    need(c->condensed, "Condense the HDG operator before applying it");
    if (c->d1()) {
        k1_hdg_apply<<<grid1(c->NT), K1_THREADS, 0, c->stream>>>(c->S, c->speeds, lam, out, c->g1);
        c->launched();
        return;
    }
    slab_trace_halo(c, lam);
    DGH_DISPATCH_N(c->n, {
        if (c->c32()) k_hdg_apply32<N><<<c->faces, 256, 0, c->stream>>>(c->S32, c->speeds, lam, out, c->basis, c->g);
        else k_hdg_apply<N><<<c->faces, 256, 0, c->stream>>>(c->S, c->speeds, lam, out, c->basis, c->g);
    });
    c->launched();
    slab_zero_ghost_faces(c, out);
}
// Face-block Jacobi blocks of the current Schur operator (FP64 or FP32 Schur blocks) into pool.
template <typename TF> void face_blocks(dgh_ctx *c, TF *pool) {
    const long long tot = (long long)c->faces * c->fw * c->fw;
    DGH_DISPATCH_N(c->n, {
        if (c->c32())
            k_face_blocks<N, TF, float><<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(c->S32, c->speeds, pool,
                                                                                              c->basis, c->g);
        else
            k_face_blocks<N, TF, double><<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(c->S, c->speeds, pool,
                                                                                               c->basis, c->g);
    });
    c->launched();
}
void op_apply(dgh_ctx *c, int op, const double *x, double *y) {
    Timed tm(c, DGH_TIMER_OPERATOR);
    if (op == DGH_OP_DG) dg_apply(c, x, y);
    else if (op == DGH_OP_DG_T) dg_apply_t(c, x, y);
    else hdg_apply(c, x, y);
}

template <int NV> void mdot_t(dgh_ctx *c, const double *V, size_t ld, int K, const double *x, const double *W, long long n) {
    k_mdot<NV><<<c->red_grid, KR_THREADS, 0, c->stream>>>(V, ld, K, x, W, n, c->partial);
}
template <int NV, int MODE>
void maxpy_t(dgh_ctx *c, const double *V, size_t ld, int K, const double *h, double *x, const double *W, long long n) {
    k_maxpy_reduce<NV, MODE><<<c->red_grid, KR_THREADS, 0, c->stream>>>(V, ld, K, h, x, W, n, c->partial);
}
template <int NV> void lincomb_t(dgh_ctx *c, const double *V, size_t ld, int K, const double *coef, double *out, long long n) {
    k_lincomb<NV><<<c->red_grid, KR_THREADS, 0, c->stream>>>(V, ld, K, coef, out, n);
}
// Arnoldi kernels are instantiated for the exact number of basis vectors (1..32), so their
// loops unroll without predicates.
#define DGH_K8(CALL, b) case b + 1: CALL(b + 1); break; case b + 2: CALL(b + 2); break; case b + 3: CALL(b + 3); break; \
    case b + 4: CALL(b + 4); break; case b + 5: CALL(b + 5); break; case b + 6: CALL(b + 6); break;              \
    case b + 7: CALL(b + 7); break; case b + 8: CALL(b + 8); break;
#define DGH_DISPATCH_K(K, CALL)                                                                 \
    switch (K) {                                                                                \
        DGH_K8(CALL, 0) DGH_K8(CALL, 8) DGH_K8(CALL, 16) DGH_K8(CALL, 24)                       \
        default: fail(DGH_ERR_INVALID, "Krylov basis too large");                               \
    }

void mdot(dgh_ctx *c, const double *V, size_t ld, int K, const double *x, const double *W, long long n, double *out) {
#define C_(NV) mdot_t<NV>(c, V, ld, K, x, W, n)
    DGH_DISPATCH_K(K, C_);
#undef C_
    k_reduce<<<K, KR_THREADS, 0, c->stream>>>(c->partial, c->red_grid, out);
    c->launched(2);
    slab_sum(c, out, K);
}
void maxpy_dot(dgh_ctx *c, const double *V, size_t ld, int K, const double *h, double *x, const double *W, long long n,
               double *out) {
#define C_(NV) maxpy_t<NV, 0>(c, V, ld, K, h, x, W, n)
    DGH_DISPATCH_K(K, C_);
#undef C_
    k_reduce<<<K, KR_THREADS, 0, c->stream>>>(c->partial, c->red_grid, out);
    c->launched(2);
    slab_sum(c, out, K);
}
void maxpy_norm(dgh_ctx *c, const double *V, size_t ld, int K, const double *h, double *x, const double *W, long long n,
                double *out) {
#define C_(NV) maxpy_t<NV, 1>(c, V, ld, K, h, x, W, n)
    DGH_DISPATCH_K(K, C_);
#undef C_
    k_reduce<<<1, KR_THREADS, 0, c->stream>>>(c->partial, c->red_grid, out);
    c->launched(2);
    slab_sum(c, out, 1);
}
void lincomb(dgh_ctx *c, const double *V, size_t ld, int K, const double *coef, double *out, long long n) {
#define C_(NV) lincomb_t<NV>(c, V, ld, K, coef, out, n)
    DGH_DISPATCH_K(K, C_);
#undef C_
    c->launched();
}
void axpby(dgh_ctx *c, double a, const double *x, double b, const double *y, double *out, long long n) {
    k_axpby<<<c->red_grid, KR_THREADS, 0, c->stream>>>(a, x, b, y, out, n);
    c->launched();
}

// gmres.cpp:17-86 with the CGS2 passes fused as dot | axpy+dot | axpy+norm.  One restart cycle
// is three segments: start (beta, V0 = r / beta, k_gmres_init), up to `restart` Arnoldi steps
// (preconditioner, operator, three sweeps, normalisation, k_gmres_update), and finish (back
// substitution, x += M^{-1} V y, true residual and its norm).  The cycle is either launched step
// by step (the host reads the device's continue flag after every step) or replayed as one CUDA
// graph whose steps are conditional nodes; the kernels and hence the numbers are the same.
struct GmresCall {
    int op;
    long long n;
    const double *W;
    double *r;
    int restart;
};
int gmres_start(dgh_ctx *c, const GmresCall &g, cudaGraphConditionalHandle h, int use_h) {
    k_wnorm2<<<c->red_grid, KR_THREADS, 0, c->stream>>>(g.r, g.W, 0, g.n, c->partial);
    k_reduce<<<1, KR_THREADS, 0, c->stream>>>(c->partial, c->red_grid, c->red + 2 * KR_MAXK);
    slab_sum(c, c->red + 2 * KR_MAXK, 1);
    k_scale_div<<<c->red_grid, KR_THREADS, 0, c->stream>>>(g.r, c->red + 2 * KR_MAXK, 1, c->V, g.n);
    k_gmres_init<<<1, 32, 0, c->stream>>>(c->gdev, c->red + 2 * KR_MAXK, h, use_h);
    c->launched(4);
    return 4;
}
int gmres_step(dgh_ctx *c, const GmresCall &g, int j, cudaGraphConditionalHandle h, int use_h) {
    const size_t ld = (size_t)c->vld;
    double *V = c->V, *w = c->gw, *z = c->gz;
    double *h1 = c->red, *h2 = c->red + KR_MAXK, *nrm = c->red + 2 * KR_MAXK;
    const int64_t before = c->launches;
    precond_apply(c, g.op, V + (size_t)j * ld, z);
    op_apply(c, g.op, z, w);
    {
        Timed tm(c, DGH_TIMER_ARNOLDI);
        mdot(c, V, ld, j + 1, w, g.W, g.n, h1);
        maxpy_dot(c, V, ld, j + 1, h1, w, g.W, g.n, h2);
        maxpy_norm(c, V, ld, j + 1, h2, w, g.W, g.n, nrm);
        k_scale_div<<<c->red_grid, KR_THREADS, 0, c->stream>>>(w, nrm, 1, V + (size_t)(j + 1) * ld, g.n);
        c->launched();
    }
    k_gmres_update<<<1, 32, 0, c->stream>>>(c->gdev, c->red, j, h, use_h);
    c->launched();
    return (int)(c->launches - before);
}
int gmres_finish(dgh_ctx *c, const GmresCall &g) {
    const int64_t before = c->launches;
    k_gmres_backsolve<<<1, 32, 0, c->stream>>>(c->gdev, c->gcoef);
    k_lincomb_dyn<<<c->red_grid, KR_THREADS, 0, c->stream>>>(c->V, (size_t)c->vld, &c->gdev->count, c->gcoef, c->gw, g.n);
    c->launched(2);
    precond_apply(c, g.op, c->gw, c->gz);
    axpby(c, 1., c->g_x, 1., c->gz, c->g_x, g.n);
    op_apply(c, g.op, c->g_x, c->gw);
    axpby(c, 1., c->g_rhs, -1., c->gw, g.r, g.n);
    k_wnorm2<<<c->red_grid, KR_THREADS, 0, c->stream>>>(g.r, g.W, 0, g.n, c->partial);
    k_reduce<<<1, KR_THREADS, 0, c->stream>>>(c->partial, c->red_grid, &c->gdev->rnorm2);
    c->launched(2);
    slab_sum(c, &c->gdev->rnorm2, 1);
    return (int)(c->launches - before);
}
// Captures one restart cycle of operator op: the start and finish segments on the context's
// stream, each Arnoldi step j inside an IF node with its own conditional handle h_j (a handle
// belongs to one conditional node), the body captured on the auxiliary stream.  The start kernel
// sets h_0 and the step-j kernel sets h_{j+1}; every handle defaults to 0 at launch, so once a
// step breaks (or does not run) all later steps are skipped.  The kernels capture their
// arguments, so the graph is rebuilt when the stage scalar 1/tau of the DG operators changes.
void build_cycle_graph(dgh_ctx *c, const GmresCall &g) {
    auto &cg = c->cycle[g.op];
    if (cg.exec) ck(cudaGraphExecDestroy(cg.exec), "cudaGraphExecDestroy");
    cg.exec = nullptr;
    if (!c->aux) ck(cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking), "cudaStreamCreate");
    const bool timing = c->timing;
    c->timing = false;  // no event records inside a captured graph
    const int64_t launches0 = c->launches;
    cudaStream_t main = c->stream;
    cudaGraph_t cap = nullptr;
    ck(cudaGraphCreate(&cap, 0), "cudaGraphCreate");
    std::vector<cudaGraphConditionalHandle> h(g.restart);
    for (auto &hj : h)
        ck(cudaGraphConditionalHandleCreate(&hj, cap, 0, cudaGraphCondAssignDefault), "cudaGraphConditionalHandleCreate");
    ck(cudaStreamBeginCaptureToGraph(main, cap, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed),
       "cudaStreamBeginCaptureToGraph");
    cudaStreamCaptureStatus st;
    int fixed = gmres_start(c, g, h[0], 1), per_step = 0;
    for (int j = 0; j < g.restart; ++j) {
        const cudaGraphNode_t *deps = nullptr;
        size_t nd = 0;
        ck(cudaStreamGetCaptureInfo(main, &st, nullptr, nullptr, &deps, &nd), "cudaStreamGetCaptureInfo");
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h[j];
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        ck(cudaGraphAddNode(&node, cap, deps, nd, &cp), "cudaGraphAddNode");
        ck(cudaStreamUpdateCaptureDependencies(main, &node, 1, cudaStreamSetCaptureDependencies),
           "cudaStreamUpdateCaptureDependencies");
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        ck(cudaStreamBeginCaptureToGraph(c->aux, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed),
           "cudaStreamBeginCaptureToGraph");
        c->stream = c->aux;
        per_step = j + 1 < g.restart ? gmres_step(c, g, j, h[j + 1], 1) : gmres_step(c, g, j, h[j], 0);
        c->stream = main;
        ck(cudaStreamEndCapture(c->aux, &body), "cudaStreamEndCapture (body)");
    }
    fixed += gmres_finish(c, g);
    ck(cudaStreamEndCapture(main, &cap), "cudaStreamEndCapture");
    ck(cudaGraphInstantiate(&cg.exec, cap, 0), "cudaGraphInstantiate");
    ck(cudaGraphDestroy(cap), "cudaGraphDestroy");
    c->timing = timing;
    c->launches = launches0;  // counted when replayed
    cg.inv_step = c->inv_step;
    cg.launches_fixed = fixed;
    cg.launches_step = per_step;
}

__global__ void k_gmres_setup(GmresDev *d, double rhs_norm, double tol, int limit, int restart) {
    if (threadIdx.x != 0) return;
    d->rhs_norm = rhs_norm;
    d->tol = tol;
    d->limit = limit;
    d->restart = restart;
    d->iters = 0;
    d->status = 0;
    d->count = 0;
}

bool lockstep_gmres(dgh_ctx *c, int op, const double *rhs, double *x, int limit, double tol, int &iters, double &rel);
void gmres(dgh_ctx *c, int op, const double *rhs, double *x, int limit, double tol, int &iters, double &rel) {
    if (c->ls && lockstep_gmres(c, op, rhs, x, limit, tol, iters, rel)) return;
    GmresCall g;
    g.op = op;
    g.n = op == DGH_OP_HDG ? c->NT : c->N;
    g.W = op == DGH_OP_HDG ? c->inv_trace_mass : c->inv_mass;
    g.restart = (int)std::min<long long>(g.n, c->cfg.restart);
    g.r = c->gres[op];
    const long long n = g.n;
    need(!c->slabbed() || op != DGH_OP_DG_T, "Slab contexts do not solve with J^T");
    ck(cudaMemcpyAsync(c->g_rhs, rhs, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream), "copy");
    if (op == DGH_OP_HDG) slab_zero_ghost_faces(c, c->g_rhs);  // a slab's Krylov vectors keep zero ghosts
    else slab_zero_ghosts(c, c->g_rhs);
    ck(cudaMemsetAsync(c->g_x, 0, n * sizeof(double), c->stream), "memset");
    ck(cudaMemcpyAsync(g.r, c->g_rhs, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream), "copy");
    const double rhs_norm = std::sqrt(std::max(0.0, c->reduce_scalar(c->g_rhs, g.W, false, n)));
    iters = 0;
    rel = 0;
    auto copy_out = [&] { ck(cudaMemcpyAsync(x, c->g_x, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream), "copy"); };
    if (rhs_norm == 0) {
        copy_out();
        return;
    }
    k_gmres_setup<<<1, 32, 0, c->stream>>>(c->gdev, rhs_norm, tol, limit, g.restart);
    c->launched();
    struct Tail {
        double rhs_norm, tol, beta, rnorm2;
        int iters, limit, count, cont, status, restart;
    };
    static_assert(sizeof(Tail) <= 4096, "pinned scratch");
    const size_t tail_off = offsetof(GmresDev, rhs_norm);
    for (;;) {
        if (c->use_graph) {
            auto &cg = c->cycle[op];
            if (!cg.exec || (op != DGH_OP_HDG && cg.inv_step != c->inv_step)) build_cycle_graph(c, g);
            ck(cudaGraphLaunch(cg.exec, c->stream), "cudaGraphLaunch");
        } else {
            gmres_start(c, g, 0, 0);
            for (int j = 0; j < g.restart; ++j) {
                ck(cudaMemcpyAsync(c->pinned, &c->gdev->cont, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "copy");
                c->sync();
                int cont = 0;
                std::memcpy(&cont, c->pinned, sizeof(int));
                if (!cont) break;
                gmres_step(c, g, j, 0, 0);
            }
            gmres_finish(c, g);
        }
        ck(cudaMemcpyAsync(c->pinned, reinterpret_cast<const char *>(c->gdev) + tail_off, sizeof(Tail),
                           cudaMemcpyDeviceToHost, c->stream), "copy");
        c->sync();
        Tail t;
        std::memcpy(&t, c->pinned, sizeof(Tail));
        if (c->use_graph)  // the graph's kernels, counted per replay
            c->launches += c->cycle[op].launches_fixed + (int64_t)t.count * c->cycle[op].launches_step;
        iters = t.iters;
        if (t.status) fail(DGH_ERR_BREAKDOWN, "GMRES Arnoldi breakdown");
        if (t.count == 0) {
            if (t.beta <= tol * rhs_norm) {
                rel = t.beta / rhs_norm;
                break;
            }
            fail(DGH_ERR_GMRES_LIMIT, "GMRES iteration limit reached");
        }
        rel = std::sqrt(std::max(0.0, t.rnorm2)) / rhs_norm;
        if (!std::isfinite(rel)) fail(DGH_ERR_NONFINITE, "Nonfinite GMRES residual");
        if (rel <= tol) break;
        if (iters >= limit) fail(DGH_ERR_GMRES_LIMIT, "GMRES iteration limit reached");
    }
    copy_out();
}

// ---- lockstep batch of DG GMRES solves ----------------------------------------------------------
// The block solves z = M^{-1} src of every gated member, one launch per factor layout.
void ls_solve_all(dgh_lockstep *L, int src, int dst, int j, int gate) {
    for (const auto &r : L->layouts) {
        if (r.key == 0)
            k_ls_solve<double, false><<<r.blocks, SOLVE_THREADS, r.smem, L->stream>>>(L->table, r.first, r.count, src, dst,
                                                                                     j, gate);
        else if (r.key == 1)
            k_ls_solve<float, false><<<r.blocks, SOLVE_THREADS, r.smem, L->stream>>>(L->table, r.first, r.count, src, dst,
                                                                                    j, gate);
        else if (r.key == 2)
            k_ls_solve<float, true><<<r.blocks, SOLVE_THREADS, r.smem, L->stream>>>(L->table, r.first, r.count, src, dst,
                                                                                   j, gate);
        else if (r.key == 3)
            k_ls_solve_half<<<r.blocks, SOLVE_THREADS, r.smem, L->stream>>>(L->table, r.first, r.count, src, dst, j, gate);
        else
            k_ls_inv_apply<<<r.blocks, INV_APPLY_THREADS, 0, L->stream>>>(L->table, r.first, r.count, src, dst, j, gate);
        L->launched();
    }
}
// dst = A src for every gated member, per degree: the face traces of src and J·v (DG, two
// launches), or the condensed Schur apply (HDG, one launch, a CTA per face).
void ls_jv_all(dgh_lockstep *L, int src, int dst, int gate) {
    for (const auto &r : L->degrees) {
        if (L->op == DGH_OP_HDG) {
            DGH_DISPATCH_N(r.key, {
                k_ls_hdg_apply<N><<<r.blocks, 256, 0, L->stream>>>(L->table, r.first, r.count, src, dst, gate);
            });
            L->launched();
            continue;
        }
        DGH_DISPATCH_N(r.key, {
            k_ls_face_trace<N><<<r.blocks, Team<N>::THREADS, 0, L->stream>>>(L->table, r.first, r.count, src, gate);
            k_ls_dg_apply<N><<<r.blocks, Team<N>::THREADS, 0, L->stream>>>(L->table, r.first, r.count, src, dst, gate);
        });
        L->launched(2);
    }
}
// The HDG members' face-block Jacobi launches from their current state (FP32 inverses or LU
// factors, chosen at each refresh): consecutive members with the same form share a launch.
void ls_plan_face_precond(dgh_lockstep *L) {
    constexpr int wpc = SOLVE_THREADS / 32;
    L->layouts.clear();
    std::vector<int> keys;
    for (int i = 0; i < (int)L->members.size(); ++i) {
        const dgh_ctx *c = L->members[i];
        const int key = c->face_inverse ? 4 : c->mixed() ? 2 : 0;
        keys.push_back(key);
        if (L->layouts.empty() || L->layouts.back().key != key) {
            dgh_lockstep::Range r;
            r.first = i;
            r.key = key;
            L->layouts.push_back(r);
        }
        auto &lr = L->layouts.back();
        L->host[i].solve0 = lr.blocks;
        L->host[i].pool = c->face_pool;
        L->host[i].perm = c->face_perm;
        lr.blocks += (c->faces + wpc - 1) / wpc;
        ++lr.count;
        if (key != 4) lr.smem = std::max(lr.smem, (key == 0 ? sizeof(double) : sizeof(float)) * (size_t)c->fw * wpc);
    }
    if (keys != L->layout_keys && L->cycle) {  // a different launch plan: capture the cycle again
        ck(cudaGraphExecDestroy(L->cycle), "cudaGraphExecDestroy");
        L->cycle = nullptr;
    }
    L->layout_keys = keys;
}
// The three segments of a lockstep restart cycle (gmres()'s start, Arnoldi step j, finish) on
// stream `st`; each returns the launches it issued.
int ls_seg_start(dgh_lockstep *L, cudaStream_t st) {
    const int cnt = (int)L->members.size();
    k_ls_wnorm2<<<L->red_total, KR_THREADS, 0, st>>>(L->table, cnt);
    k_ls_reduce<<<cnt, KR_THREADS, 0, st>>>(L->table, cnt, 1, 2, 0);
    k_ls_scale_div<<<L->red_total, KR_THREADS, 0, st>>>(L->table, cnt, LS_R, LS_VJ, 0, 0);
    k_ls_gmres_init<<<cnt, 32, 0, st>>>(L->table);
    L->launched(4);
    return 4;
}
int ls_seg_step(dgh_lockstep *L, cudaStream_t st, int j) {
    const int cnt = (int)L->members.size();
    const int64_t before = L->launches;
    cudaStream_t keep = L->stream;
    L->stream = st;
    ls_solve_all(L, LS_VJ, LS_Z, j, 1);
    ls_jv_all(L, LS_Z, LS_W, 1);
    L->stream = keep;
    const int K = j + 1;
#define C_(NV) k_ls_mdot<NV><<<L->red_total, KR_THREADS, 0, st>>>(L->table, cnt, K)
    DGH_DISPATCH_K(K, C_);
#undef C_
    k_ls_reduce<<<cnt * K, KR_THREADS, 0, st>>>(L->table, cnt, K, 0, 1);
#define C_(NV) k_ls_maxpy<NV, 0><<<L->red_total, KR_THREADS, 0, st>>>(L->table, cnt, K)
    DGH_DISPATCH_K(K, C_);
#undef C_
    k_ls_reduce<<<cnt * K, KR_THREADS, 0, st>>>(L->table, cnt, K, 1, 1);
#define C_(NV) k_ls_maxpy<NV, 1><<<L->red_total, KR_THREADS, 0, st>>>(L->table, cnt, K)
    DGH_DISPATCH_K(K, C_);
#undef C_
    k_ls_reduce<<<cnt, KR_THREADS, 0, st>>>(L->table, cnt, 1, 2, 1);
    k_ls_scale_div<<<L->red_total, KR_THREADS, 0, st>>>(L->table, cnt, LS_W, LS_VJ1, j, 1);
    k_ls_gmres_update<<<cnt, 32, 0, st>>>(L->table, j);
    L->launched(8);
    return (int)(L->launches - before);
}
int ls_seg_finish(dgh_lockstep *L, cudaStream_t st) {
    const int cnt = (int)L->members.size();
    const int64_t before = L->launches;
    cudaStream_t keep = L->stream;
    L->stream = st;
    k_ls_gmres_backsolve<<<cnt, 32, 0, st>>>(L->table);
    k_ls_lincomb<<<L->red_total, KR_THREADS, 0, st>>>(L->table, cnt);
    L->launched(2);
    ls_solve_all(L, LS_W, LS_Z, 0, 0);
    k_ls_axpby<<<L->red_total, KR_THREADS, 0, st>>>(L->table, cnt, 1., LS_X, 1., LS_Z, LS_X);
    L->launched();
    ls_jv_all(L, LS_X, LS_W, 0);
    k_ls_axpby<<<L->red_total, KR_THREADS, 0, st>>>(L->table, cnt, 1., LS_RHS, -1., LS_W, LS_R);
    k_ls_wnorm2<<<L->red_total, KR_THREADS, 0, st>>>(L->table, cnt);
    k_ls_reduce<<<cnt, KR_THREADS, 0, st>>>(L->table, cnt, 1, 3, 0);
    k_ls_tails<<<(cnt + 127) / 128, 128, 0, st>>>(L->table, cnt, L->tails);
    L->launched(4);
    L->stream = keep;
    return (int)(L->launches - before);
}
// Captures one lockstep restart cycle as a CUDA graph: the start segment, one IF node per
// Arnoldi step whose handle the preceding k_ls_cont_cond sets (any member continues), the finish
// segment; the step bodies are captured on the auxiliary stream (as build_cycle_graph does for
// one context).
void ls_build_graph(dgh_lockstep *L) {
    const int cnt = (int)L->members.size();
    if (!L->aux) ck(cudaStreamCreateWithFlags(&L->aux, cudaStreamNonBlocking), "cudaStreamCreate");
    const int64_t launches0 = L->launches;
    cudaGraph_t cap = nullptr;
    ck(cudaGraphCreate(&cap, 0), "cudaGraphCreate");
    std::vector<cudaGraphConditionalHandle> h(L->restart);
    for (auto &hj : h)
        ck(cudaGraphConditionalHandleCreate(&hj, cap, 0, cudaGraphCondAssignDefault), "cudaGraphConditionalHandleCreate");
    ck(cudaStreamBeginCaptureToGraph(L->stream, cap, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed),
       "cudaStreamBeginCaptureToGraph");
    int fixed = ls_seg_start(L, L->stream), per_step = 0;
    k_ls_cont_cond<<<1, 1024, 0, L->stream>>>(L->table, cnt, h[0]);
    L->launched();
    ++fixed;
    cudaStreamCaptureStatus stc;
    for (int j = 0; j < L->restart; ++j) {
        const cudaGraphNode_t *deps = nullptr;
        size_t nd = 0;
        ck(cudaStreamGetCaptureInfo(L->stream, &stc, nullptr, nullptr, &deps, &nd), "cudaStreamGetCaptureInfo");
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h[j];
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        ck(cudaGraphAddNode(&node, cap, deps, nd, &cp), "cudaGraphAddNode");
        ck(cudaStreamUpdateCaptureDependencies(L->stream, &node, 1, cudaStreamSetCaptureDependencies),
           "cudaStreamUpdateCaptureDependencies");
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        ck(cudaStreamBeginCaptureToGraph(L->aux, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed),
           "cudaStreamBeginCaptureToGraph");
        per_step = ls_seg_step(L, L->aux, j);
        if (j + 1 < L->restart) {
            k_ls_cont_cond<<<1, 1024, 0, L->aux>>>(L->table, cnt, h[j + 1]);
            L->launched();
            ++per_step;
        }
        ck(cudaStreamEndCapture(L->aux, &body), "cudaStreamEndCapture (body)");
    }
    fixed += ls_seg_finish(L, L->stream);
    ck(cudaStreamEndCapture(L->stream, &cap), "cudaStreamEndCapture");
    ck(cudaGraphInstantiate(&L->cycle, cap, 0), "cudaGraphInstantiate");
    ck(cudaGraphDestroy(cap), "cudaGraphDestroy");
    L->launches = launches0;  // counted when replayed
    L->graph_fixed = fixed;
    L->graph_step = per_step;
}
// One session's lockstep solve: gmres() of every live member, restart cycle by restart cycle
// and Arnoldi step by Arnoldi step, each phase one launch over the members.  Stepped, the host
// reads one continue flag per member after each step; replayed (when every member replays its
// own cycles as graphs), each cycle is one graph launch whose steps are conditional on any
// member continuing.  After each cycle the host reads one tail record per member and applies
// gmres()'s stopping and failure rules per member.
void ls_run(dgh_lockstep *L) {
    const int cnt = (int)L->members.size();
    cudaStream_t gs = L->stream;
    bool any = false, graph = true;
    for (int i = 0; i < cnt; ++i) {
        auto &sl = L->slots[i];
        const bool live = sl.arrived && !sl.trivial && sl.code == DGH_OK;
        L->host[i].live = live ? 1 : 0;
        L->host[i].inv_step = L->members[i]->inv_step;
        if (live) ck(cudaStreamWaitEvent(gs, sl.ready, 0), "cudaStreamWaitEvent");
        any = any || live;
        graph = graph && L->members[i]->use_graph;
    }
    if (!any) return;
    ++L->sessions;
    if (L->op == DGH_OP_HDG) ls_plan_face_precond(L);
    if (graph && !L->cycle) ls_build_graph(L);
    const size_t tb = sizeof(LsMember) * (size_t)cnt;
    for (;;) {
        ck(cudaMemcpyAsync(L->table, L->host, tb, cudaMemcpyHostToDevice, gs), "copy member table");
        ++L->cycles;
        if (graph) {
            ck(cudaGraphLaunch(L->cycle, gs), "cudaGraphLaunch");
        } else {
            ls_seg_start(L, gs);
            for (int j = 0; j < L->restart; ++j) {
                k_ls_cont<<<(cnt + 127) / 128, 128, 0, gs>>>(L->table, cnt, L->flags);
                L->launched();
                ck(cudaMemcpyAsync(L->flags_host, L->flags, sizeof(int) * cnt, cudaMemcpyDeviceToHost, gs), "copy flags");
                ck(cudaStreamSynchronize(gs), "cudaStreamSynchronize");
                bool cont = false;
                for (int i = 0; i < cnt; ++i) cont = cont || L->flags_host[i];
                if (!cont) break;
                ++L->steps;
                ls_seg_step(L, gs, j);
            }
            ls_seg_finish(L, gs);
        }
        ck(cudaMemcpyAsync(L->tails_host, L->tails, sizeof(LsTail) * cnt, cudaMemcpyDeviceToHost, gs), "copy tails");
        ck(cudaStreamSynchronize(gs), "cudaStreamSynchronize");
        if (graph) {  // the replayed steps: as many as the longest member's basis this cycle
            int taken = 0;
            for (int i = 0; i < cnt; ++i)
                if (L->host[i].live) taken = std::max(taken, L->tails_host[i].count);
            L->steps += taken;
            L->launches += L->graph_fixed + (int64_t)taken * L->graph_step;
        }
        bool more = false;
        for (int i = 0; i < cnt; ++i) {
            if (!L->host[i].live) continue;
            auto &sl = L->slots[i];
            const LsTail &t = L->tails_host[i];
            sl.iters = t.iters;
            bool done = false;
            auto failed = [&](int code, const char *msg) {
                sl.code = code;
                sl.msg = msg;
                done = true;
            };
            if (t.status) failed(DGH_ERR_BREAKDOWN, "GMRES Arnoldi breakdown");
            else if (t.count == 0) {
                if (t.beta <= sl.tol * sl.rhs_norm) {
                    sl.rel = t.beta / sl.rhs_norm;
                    done = true;
                } else failed(DGH_ERR_GMRES_LIMIT, "GMRES iteration limit reached");
            } else {
                sl.rel = std::sqrt(std::max(0.0, t.rnorm2)) / sl.rhs_norm;
                if (!std::isfinite(sl.rel)) failed(DGH_ERR_NONFINITE, "Nonfinite GMRES residual");
                else if (sl.rel <= sl.tol) done = true;
                else if (sl.iters >= sl.limit) failed(DGH_ERR_GMRES_LIMIT, "GMRES iteration limit reached");
            }
            if (done) L->host[i].live = 0;
            more = more || !done;
        }
        if (!more) break;
    }
}
// Ends a session: the last arrival (or withdrawal) runs the lockstep solve, then wakes the others.
void ls_complete(dgh_lockstep *L) {
    try {
        ls_run(L);
    } catch (const Failure &e) {
        for (auto &sl : L->slots)
            if (sl.arrived && sl.code == DGH_OK) {
                sl.code = e.code;
                sl.msg = e.message;
            }
    } catch (const std::exception &e) {
        for (auto &sl : L->slots)
            if (sl.arrived && sl.code == DGH_OK) {
                sl.code = DGH_ERR_CUDA;
                sl.msg = e.what();
            }
    }
    cudaEventRecord(L->finished, L->stream);
    std::lock_guard<std::mutex> lk(L->mu);
    L->open = false;
    ++L->generation;
    L->cv.notify_all();
}
void ls_arrive(dgh_lockstep *L, int idx) {
    std::unique_lock<std::mutex> lk(L->mu);
    const uint64_t gen = L->generation;
    L->slots[idx].arrived = true;
    ++L->arrived;
    if (L->arrived + L->withdrawn == L->expected) {
        lk.unlock();
        ls_complete(L);
        return;
    }
    L->cv.wait(lk, [&] { return L->generation != gen; });
}
// gmres() of op DG for a member of an open session: the solve's own copies and |rhs| on the
// member's stream, then the rendezvous; false when the context has no open session to join.
bool lockstep_gmres(dgh_ctx *c, int op, const double *rhs, double *x, int limit, double tol, int &iters, double &rel) {
    dgh_lockstep *L = c->ls;
    if (op != L->op) return false;
    {
        std::lock_guard<std::mutex> lk(L->mu);
        if (!L->open) return false;
        const auto &sl = L->slots[c->ls_index];
        if (sl.arrived || sl.withdrawn) return false;  // one solve per member and session
    }
    auto &sl = L->slots[c->ls_index];
    const long long n = op == DGH_OP_HDG ? c->NT : c->N;
    double *r = c->gres[op];
    ck(cudaMemcpyAsync(c->g_rhs, rhs, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream), "copy");
    ck(cudaMemsetAsync(c->g_x, 0, n * sizeof(double), c->stream), "memset");
    ck(cudaMemcpyAsync(r, c->g_rhs, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream), "copy");
    const double *W = op == DGH_OP_HDG ? c->inv_trace_mass : c->inv_mass;
    const double rhs_norm = std::sqrt(std::max(0.0, c->reduce_scalar(c->g_rhs, W, false, n)));
    sl.tol = tol;
    sl.limit = limit;
    sl.rhs_norm = rhs_norm;
    sl.trivial = rhs_norm == 0;
    sl.iters = 0;
    sl.rel = 0;
    sl.code = DGH_OK;
    sl.msg.clear();
    if (!sl.trivial) {
        k_gmres_setup<<<1, 32, 0, c->stream>>>(c->gdev, rhs_norm, tol, limit, (int)std::min<long long>(n, c->cfg.restart));
        c->launched();
    }
    ck(cudaEventRecord(sl.ready, c->stream), "cudaEventRecord");
    ls_arrive(L, c->ls_index);
    if (sl.code != DGH_OK) fail(sl.code, sl.msg);
    ck(cudaStreamWaitEvent(c->stream, L->finished, 0), "cudaStreamWaitEvent");
    iters = sl.iters;
    rel = sl.rel;
    ck(cudaMemcpyAsync(x, c->g_x, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream), "copy");
    return true;
}

void build_rule(dgh_ctx *c) {
    ErrorRule h{};
    std::vector<double> ex, ew;
    const int Q = std::max(20, 2 * c->n + 3);
    gauss_rule(Q, ex, ew);
    h.Q = Q;
    for (int q = 0; q < Q; ++q) {
        h.ex[q] = ex[q];
        h.ew[q] = ew[q];
        auto v = lagrange(c->xnodes, ex[q]);
        for (int i = 0; i < c->n; ++i) h.ev[q * c->n + i] = v[i];
    }
    for (int i = 0; i < c->n; ++i)
        for (int q = 0; q < Q; ++q) h.proj[i * Q + q] = h.ev[q * c->n + i] * ew[q] / c->basis.w[i];
    c->rule = c->alloc<ErrorRule>(1);
    ck(cudaMemcpy(c->rule, &h, sizeof(h), cudaMemcpyHostToDevice), "upload rule");
}

__global__ void k_fill_mass(double *mass, double *inv_mass, Basis1D b, Grid g, int n, long long N) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int P = n * n, node = (int)(i % P), ix = node % n, iy = node / n;
    const double m = .25 * g.hx * g.hy * b.w[ix] * b.w[iy];
    mass[i] = m;
    inv_mass[i] = 1 / m;
}
__global__ void k_fill_trace_mass(double *inv_tm, Basis1D b, Grid g, int n, long long NT) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NT) return;
    const int fw = 4 * n, face = (int)(i / fw), q = (int)(i % fw) % n;
    inv_tm[i] = 1 / face_weight(g, b, face, q);
}

// block_ilu.cpp:15-45 on BlockGraph::periodic(rows) (block_graph.cpp:7-19,30-35): each row's
// columns {row-1, row, row+1} sorted and unique, the diagonal slots and, for every block left of
// the diagonal, the (target, upper) pairs its elimination updates; uploaded once.
void build_ilu_plan(dgh_ctx *c, dgh_ctx::IluPlan &pl, int rows, int m) {
    std::vector<int> row_ptr(rows + 1, 0), col, diag(rows), slot_row;
    for (int r = 0; r < rows; ++r) {
        std::vector<int> cols = {(r + rows - 1) % rows, r, (r + 1) % rows};
        std::sort(cols.begin(), cols.end());
        cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
        for (int cc : cols) {
            col.push_back(cc);
            slot_row.push_back(r);
        }
        row_ptr[r + 1] = (int)col.size();
    }
    auto find = [&](int r, int cc) {
        for (int p = row_ptr[r]; p < row_ptr[r + 1]; ++p)
            if (col[p] == cc) return p;
        return -1;
    };
    std::vector<int> off(col.size() + 1, 0), target, upper;
    for (int r = 0; r < rows; ++r) {
        diag[r] = find(r, r);
        for (int slot = row_ptr[r]; slot < row_ptr[r + 1]; ++slot) {
            off[slot] = (int)target.size();
            const int elim = col[slot];
            if (elim >= r) continue;
            for (int u = row_ptr[elim]; u < row_ptr[elim + 1]; ++u) {
                if (col[u] <= elim) continue;
                const int t = find(r, col[u]);
                if (t >= 0) {
                    target.push_back(t);
                    upper.push_back(u);
                }
            }
        }
    }
    off.back() = (int)target.size();
    auto upload = [&](const std::vector<int> &h) {
        int *d = c->alloc<int>(std::max<size_t>(h.size(), 1));
        if (!h.empty()) ck(cudaMemcpy(d, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice), "upload pattern");
        return d;
    };
    pl.rows = rows;
    pl.m = m;
    pl.nnz = (int)col.size();
    pl.row_ptr = upload(row_ptr);
    pl.col = upload(col);
    pl.diag = upload(diag);
    pl.slot_row = upload(slot_row);
    pl.upd_off = upload(off);
    pl.upd_target = upload(target);
    pl.upd_upper = upload(upper);
    pl.perm = c->alloc<int>((size_t)rows * m);
    pl.vals = c->alloc<char>((size_t)pl.nnz * m * m * (c->mixed() ? sizeof(float) : sizeof(double)));
}

// Sizes, reference element and pools of a 1D context (dg_hdg_1d/src/discretization.cpp:4-14,
// nodal_basis.hpp:34-65 with its separate quadrature rule).  Called after the stream exists.
void create1(dgh_ctx *c, const dgh_config &k) {
    const int n = k.degree + 1, Q = k.quadrature ? k.quadrature : n;
    c->dim = 1;
    c->n = n;
    c->Q = Q;
    c->P = n;
    c->m = NV1 * n;
    c->cells = k.nx;
    c->faces = k.nx;
    c->fw = NV1;
    c->t = T1;
    c->N = (long long)c->cells * c->m;
    c->NT = (long long)c->faces * NV1;
    c->nspeeds = 2 * (size_t)c->faces;
    c->cs.kind = 2;  // the unrotated simple wave: exact_state's axis case with y unused
    c->cs.cosine = 1.;
    c->cs.sine = 0.;
    c->cs.lx = 2.;
    c->cs.ly = 1.;
    c->cs.gamma = 3.;
    c->g1.cells = c->cells;
    c->g1.h = 2.0 / c->cells;
    c->g1.gamma = 3.;
    c->g.nx = c->cells;
    c->g.ny = 1;
    c->g.cells = c->cells;
    c->g.hx = c->g1.h;
    c->g.hy = 1.;
    c->g.gamma = 3.;
    std::vector<double> x, w, qx, qw;
    gauss_rule(n, x, w);
    gauss_rule(Q, qx, qw);
    c->xnodes = x;
    std::vector<double> bary(n, 1.), D(n * n, 0.);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            if (i != j) bary[i] /= x[i] - x[j];
    for (int i = 0; i < n; ++i) {
        double s = 0;
        for (int j = 0; j < n; ++j)
            if (i != j) {
                D[i * n + j] = bary[j] / (bary[i] * (x[i] - x[j]));
                s += D[i * n + j];
            }
        D[i * n + i] = -s;
    }
    auto eL = lagrange(x, -1.), eR = lagrange(x, 1.);
    Basis1Q &b = c->b1;
    b.n = n;
    b.Q = Q;
    b.colloc = Q == n;
    for (int i = 0; i < n; ++i) {
        b.w[i] = c->basis.w[i] = w[i];
        b.eL[i] = c->basis.eL[i] = eL[i];
        b.eR[i] = c->basis.eR[i] = eR[i];
    }
    for (int q = 0; q < Q; ++q) {
        const auto v = lagrange(x, qx[q]);
        for (int i = 0; i < n; ++i) b.values[q * n + i] = b.colloc ? (q == i ? 1. : 0.) : v[i];
    }
    for (int q = 0; q < Q; ++q)
        for (int i = 0; i < n; ++i) {
            double s = 0;
            for (int j = 0; j < n; ++j) s += b.values[q * n + j] * D[j * n + i];
            b.wd[q * n + i] = qw[q] * s;
        }
    c->old = c->alloc<double>(c->N);
    c->mass = c->alloc<double>(c->N);
    c->inv_mass = c->alloc<double>(c->N);
    c->inv_trace_mass = c->alloc<double>(c->NT);
    c->speeds = c->alloc<double>(c->nspeeds);
    c->traces = c->alloc<double>((size_t)c->cells * T1);
    c->traces2 = c->alloc<double>((size_t)c->cells * T1);
    c->partial = c->alloc<double>((size_t)std::max<long long>(KR_MAXK * c->red_grid, 4LL * c->cells + 64));
    c->red = c->alloc<double>(4 * KR_MAXK);
    c->vol = c->alloc<double>((size_t)c->cells * Q * 9);
    c->fcache = c->alloc<double>((size_t)c->faces * 18);
    c->status = c->alloc<int>(1);
    c->ok = c->alloc<int>(1);
    ck(cudaMemset(c->status, 0, sizeof(int)), "memset");
    build_rule(c);
    k1_fill_mass<<<grid1(c->N, 256), 256, 0, c->stream>>>(c->mass, c->inv_mass, c->inv_trace_mass, c->b1, c->g1, n);
    c->launched();
    const size_t tsz = c->mixed() ? sizeof(float) : sizeof(double);
    if (c->has_dg()) {
        c->dg_pool = c->alloc<char>((size_t)c->cells * c->m * c->m * tsz);
        c->dg_perm = c->alloc<int>((size_t)c->cells * c->m);
    }
    if (c->has_hdg()) {
        c->S = c->alloc<double>((size_t)c->cells * T1 * T1);
        c->X = c->alloc<double>((size_t)c->cells * c->m * T1);
        c->Y = c->alloc<double>((size_t)c->cells * c->m);
        c->cy = c->alloc<double>((size_t)c->cells * T1);
        c->hrhs = c->alloc<double>(c->NT);
        const size_t per_cell = (size_t)c->m * (c->m + T1 + 1) * sizeof(double);
        const size_t budget = (size_t)8 << 30;
        c->aug_cells = (int)std::max<size_t>(1, std::min<size_t>(c->cells, budget / per_cell));
        c->aug = c->alloc<double>((size_t)c->aug_cells * c->m * (c->m + T1 + 1));
        c->aug_perm = c->alloc<int>((size_t)c->aug_cells * c->m);
        c->face_pool = c->alloc<char>((size_t)c->faces * NV1 * NV1 * tsz);
        c->face_perm = c->alloc<int>((size_t)c->faces * NV1);
    }
    if (c->ilu()) {
        if (c->has_dg()) build_ilu_plan(c, c->ilu_dg, c->cells, c->m);
        if (c->has_hdg()) build_ilu_plan(c, c->ilu_hdg, c->faces, NV1);
    }
    const long long vn = std::max(c->has_dg() ? c->N : 0LL, c->has_hdg() ? c->NT : 0LL);
    c->vld = ((vn + 31) / 32) * 32;
    c->restart = k.restart;
    c->V = c->alloc<double>((size_t)c->vld * (k.restart + 1));
    c->gw = c->alloc<double>(vn);
    c->gz = c->alloc<double>(vn);
    if (c->has_dg()) {
        c->gres[DGH_OP_DG] = c->alloc<double>(c->N);
        c->gres[DGH_OP_DG_T] = c->alloc<double>(c->N);
    }
    if (c->has_hdg()) c->gres[DGH_OP_HDG] = c->alloc<double>(c->NT);
    c->gcoef = c->alloc<double>(KR_MAXK);
    c->g_rhs = c->alloc<double>(vn);
    c->g_x = c->alloc<double>(vn);
    c->gdev = c->alloc<GmresDev>(1);
    ck(cudaMemset(c->V, 0, sizeof(double) * (size_t)c->vld * (k.restart + 1)), "memset");
    c->sync();
}
}  // namespace

// ============================================================================ C ABI
extern "C" {

void dgh_config_default(dgh_config *c) {
    std::memset(c, 0, sizeof(*c));
    c->nx = 8; c->ny = 8; c->degree = 3; c->quadrature = 0;
    c->restart = 30; c->max_linear = 1500; c->max_newton = 30; c->steps = 0;
    c->newton_steps = 0; c->warmup_updates = 0;
    c->cfl = 2.; c->final_time = .2; c->safety = 1.1;
    c->nonlinear_tolerance = 1e-12; c->linear_tolerance = 1e-12;
    c->method = DGH_METHOD_BOTH; c->integrator = DGH_INTEGRATOR_DIRK3; c->testcase = DGH_TEST_DIAGONAL;
    c->precision = DGH_PRECISION_FP64; c->check_update = 0; c->device = 0; c->dim = 2;
}

static thread_local std::string g_create_error;

}  // extern "C"

namespace {
// The mesh rows of a slab context (dgh_ctx_create_slab), and of every other context none.
struct SlabInit {
    dgh_comm *comm = nullptr;
    int row0 = 0, rows = 0, ny = 0;
};
int create_ctx(const dgh_config *cfg, const SlabInit *slab, dgh_ctx **out);
}  // namespace

extern "C" {
int dgh_ctx_create(const dgh_config *cfg, dgh_ctx **out) { return create_ctx(cfg, nullptr, out); }

int dgh_ctx_create_slab(const dgh_config *cfg, dgh_comm *comm, dgh_ctx **out) {
    if (!cfg || !out) return DGH_ERR_INVALID;
    *out = nullptr;
    const char *why = nullptr;
    if (!comm) why = "null communicator";
    else if (cfg->dim != 2 || cfg->method == DGH_METHOD_BOTH)
        why = "Slab decomposition is built for the 2D DG or HDG method";
    else if (cfg->quadrature != 0 && cfg->quadrature != cfg->degree + 1)
        why = "Slab decomposition is built for the collocated volume rule";
    else if (cfg->preconditioner != 0) why = "Slab decomposition is built for the block-Jacobi preconditioner";
    else if (cfg->ny < 3 || comm->size > cfg->ny) why = "Slab decomposition needs at least one mesh row per rank";
    else if (cfg->method == DGH_METHOD_HDG && cfg->ny < 2 * comm->size)
        why = "HDG slabs need at least two mesh rows per rank";
    if (why) {
        g_create_error = why;
        return DGH_ERR_INVALID;
    }
    SlabInit si;
    si.comm = comm;
    si.ny = cfg->ny;
    dgh_slab::rows_of(cfg->ny, comm->size, comm->rank, si.row0, si.rows);
    dgh_config local = *cfg;
    local.ny = si.rows + 1 + (cfg->method == DGH_METHOD_HDG ? 2 : 1);  // the slab's rows with its ghost rows
    return create_ctx(&local, &si, out);
}

int dgh_slab_info(const dgh_ctx *c, int64_t out[8]) {
    if (!c || !out || !c->slabbed()) return DGH_ERR_INVALID;
    out[0] = c->slab.row0;
    out[1] = c->slab.rows;
    out[2] = c->slab.comm->rank;
    out[3] = c->slab.comm->size;
    out[4] = c->slab.row_len;
    out[5] = (int64_t)c->slab.rows * c->slab.row_len;
    out[6] = c->slab.above;
    out[7] = c->slab.face_row;
    return DGH_OK;
}
}  // extern "C"

namespace {
int create_ctx(const dgh_config *cfg, const SlabInit *slab, dgh_ctx **out) {
    if (!cfg || !out) return DGH_ERR_INVALID;
    *out = nullptr;
    dgh_ctx *c = new dgh_ctx;
    c->cfg = *cfg;
    const int rc = guard(c, [&] {
        const dgh_config &k = *cfg;
        need(k.dim == 1 || k.dim == 2, "Invalid dimension (1 or 2)");
        need(k.preconditioner == 0 || k.preconditioner == 1, "Invalid block preconditioner");
        need(k.preconditioner == 0 || k.dim == 1 || k.method == DGH_METHOD_DG,
             "2D block ILU(0) is built for the DG operator only (method dg)");
        need(k.condense32 == 0 || (k.condense32 == 1 && k.dim == 2), "FP32 condensation is a 2D HDG option (0 or 1)");
        need(k.forcing == 0 || k.forcing == 1, "Invalid forcing (0 or 1)");
        // config.cpp:6-22 (dg_hdg_1d/src/config.cpp:6-21 in 1D)
        need(k.nx >= 3 && (k.dim == 1 || k.ny >= 3) && k.degree >= 0 && k.degree <= 8 && k.quadrature >= 0,
             "Invalid mesh or degree");
        need(k.quadrature == 0 || k.quadrature >= k.degree + 1, "Quadrature must be >= degree+1");
        if (k.dim == 2)
            need(k.quadrature <= MAXQ2, "Quadrature above 16 points is not supported on the device (2D)");
        else
            need(k.quadrature <= MAXQ1, "Quadrature above 20 points is not supported on the device");
        need(k.restart > 0 && k.max_linear > 0 && k.max_newton > 0 && k.steps >= 0, "Invalid iteration limit");
        need(k.newton_steps >= 0 && k.warmup_updates >= 0, "Invalid timing update count");
        need(std::isfinite(k.cfl) && k.cfl > 0 && std::isfinite(k.final_time) && k.final_time >= 0,
             "CFL must be positive and final time nonnegative");
        need(std::isfinite(k.safety) && k.safety >= 1 && std::isfinite(k.nonlinear_tolerance) &&
                 k.nonlinear_tolerance > 0 && std::isfinite(k.linear_tolerance) && k.linear_tolerance > 0 &&
                 k.linear_tolerance < 1,
             "Invalid solver tolerance or wave-speed safety");
        need(k.method >= 0 && k.method <= 2, "Method must be dg, hdg, or both");
        need(k.dim == 1 || (k.testcase >= 0 && k.testcase <= 2), "Invalid testcase");
        need(k.precision >= 0 && k.precision <= 2, "Invalid precision");
        need(k.precision != DGH_PRECISION_MIXED16 || k.dim == 2, "FP16 factor storage is a 2D option");
        need(k.restart <= KR_MAXK - 1, "restart must be at most 31 on the device GMRES");
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) fail(DGH_ERR_CUDA, "no CUDA device available");
        ck(cudaSetDevice(k.device), "cudaSetDevice");
        cudaDeviceProp prop{};
        ck(cudaGetDeviceProperties(&prop, k.device), "cudaGetDeviceProperties");
        if (prop.major < 10) fail(DGH_ERR_CUDA, "this library is built for sm_100a (B200) only");
        c->sms = prop.multiProcessorCount;
        c->red_grid = c->sms * RED_BLOCKS_PER_SM;
        ck(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        ck(cudaMallocHost((void **)&c->pinned, 4096), "cudaMallocHost");
        if (k.dim == 1) {
            create1(c, k);
            return;
        }

        c->n = k.degree + 1;
        c->P = c->n * c->n;
        c->m = NVAR * c->P;
        c->cells = k.nx * k.ny;
        c->faces = 2 * c->cells;
        c->fw = NVAR * c->n;
        c->t = NFACES * c->fw;
        c->N = (long long)c->cells * c->m;
        c->NT = (long long)c->faces * c->fw;
        c->Q = k.quadrature ? k.quadrature : c->n;
        c->nspeeds = 2 * (size_t)c->faces * c->n;
        // example.hpp:9-14
        const double pi = std::acos(-1.);
        c->cs.kind = k.testcase == DGH_TEST_DIAGONAL ? 0 : (k.testcase == DGH_TEST_WAVE ? 1 : 2);
        c->cs.cosine = std::cos(45. * pi / 180.);
        c->cs.sine = std::sin(45. * pi / 180.);
        c->cs.lx = c->cs.kind == 0 ? 2. / c->cs.cosine : 2.;
        c->cs.ly = c->cs.kind == 0 ? 2. / c->cs.sine : 2.;
        c->cs.gamma = 3.;
        c->g.nx = k.nx;
        c->g.ny = k.ny;
        c->g.cells = c->cells;
        c->g.hx = c->cs.lx / k.nx;
        c->g.hy = c->cs.ly / (slab ? slab->ny : k.ny);
        c->g.gamma = 3.;
        if (slab) {
            c->slab.comm = slab->comm;
            c->slab.row0 = slab->row0;
            c->slab.rows = slab->rows;
            c->slab.ny = slab->ny;
            c->slab.above = k.ny - 1 - slab->rows;
            c->slab.row_len = (long long)k.nx * NVAR * c->n * c->n;
            c->slab.face_row = (long long)k.nx * c->fw;
            c->slab.vol = dgh_slab::volume_plan(c->slab.row_len, slab->rows, c->slab.above);
            c->slab.trace = dgh_slab::trace_plan(c->slab.face_row, (long long)c->cells * c->fw, slab->rows);
        }
        // nodal_basis.hpp:34-65
        std::vector<double> x, w;
        gauss_rule(c->n, x, w);
        c->xnodes = x;
        const int n = c->n;
        std::vector<double> bary(n, 1.);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                if (i != j) bary[i] /= x[i] - x[j];
        std::vector<double> D(n * n, 0.);
        for (int i = 0; i < n; ++i) {
            double s = 0;
            for (int j = 0; j < n; ++j)
                if (i != j) {
                    D[i * n + j] = bary[j] / (bary[i] * (x[i] - x[j]));
                    s += D[i * n + j];
                }
            D[i * n + i] = -s;
        }
        auto eL = lagrange(x, -1.), eR = lagrange(x, 1.);
        for (int i = 0; i < n; ++i) {
            c->basis.w[i] = w[i];
            c->basis.eL[i] = eL[i];
            c->basis.eR[i] = eR[i];
        }
        for (int q = 0; q < n; ++q)
            for (int i = 0; i < n; ++i) c->basis.dw[q * n + i] = w[q] * D[q * n + i];

        // ---- pools (sized once; nothing else allocates on the hot path)
        c->old = c->alloc<double>(c->N);
        c->mass = c->alloc<double>(c->N);
        c->inv_mass = c->alloc<double>(c->N);
        c->inv_trace_mass = c->alloc<double>(c->NT);
        c->speeds = c->alloc<double>(2 * (size_t)c->faces * n);
        c->traces = c->alloc<double>((size_t)c->cells * NFACES * n * NVAR);
        c->traces2 = c->alloc<double>((size_t)c->cells * NFACES * n * NVAR);
        c->partial = c->alloc<double>((size_t)std::max<long long>(KR_MAXK * c->red_grid, 4LL * c->cells + 64));
        c->red = c->alloc<double>(4 * KR_MAXK);
        c->vol = c->alloc<double>((size_t)c->cells * c->P * 3);
        c->fcache = c->alloc<double>((size_t)c->faces * n * 8);
        c->status = c->alloc<int>(1);
        c->ok = c->alloc<int>(1);
        ck(cudaMemset(c->status, 0, sizeof(int)), "memset");
        build_rule(c);
        if (c->overint()) {
            // nodal_basis.hpp:37-56: the volume rule's values and weighted derivatives
            BasisQ h{};
            h.Q = c->Q;
            std::vector<double> qx, qw, bary(n, 1.), D(n * n, 0.);
            gauss_rule(c->Q, qx, qw);
            const auto &xn = c->xnodes;
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j)
                    if (i != j) bary[i] /= xn[i] - xn[j];
            for (int i = 0; i < n; ++i) {
                double sum = 0;
                for (int j = 0; j < n; ++j)
                    if (i != j) {
                        D[i * n + j] = bary[j] / (bary[i] * (xn[i] - xn[j]));
                        sum += D[i * n + j];
                    }
                D[i * n + i] = -sum;
            }
            for (int q = 0; q < c->Q; ++q) {
                const auto v = lagrange(xn, qx[q]);
                for (int i = 0; i < n; ++i) h.V[q * n + i] = v[i];
                h.qw[q] = qw[q];
            }
            for (int q = 0; q < c->Q; ++q)
                for (int i = 0; i < n; ++i) {
                    double sum = 0;
                    for (int kk = 0; kk < n; ++kk) sum += h.V[q * n + kk] * D[kk * n + i];
                    h.wd[q * n + i] = qw[q] * sum;
                }
            c->bq = c->alloc<BasisQ>(1);
            ck(cudaMemcpy(c->bq, &h, sizeof(BasisQ), cudaMemcpyHostToDevice), "upload volume rule");
            c->volq = c->alloc<double>((size_t)c->cells * c->Q * c->Q * 3);
        }
        c->basis_dev = c->alloc<Basis1D>(1);
        ck(cudaMemcpy(c->basis_dev, &c->basis, sizeof(Basis1D), cudaMemcpyHostToDevice), "upload basis");
        const int tb = 256;
        k_fill_mass<<<(unsigned)((c->N + tb - 1) / tb), tb, 0, c->stream>>>(c->mass, c->inv_mass, c->basis, c->g, n, c->N);
        k_fill_trace_mass<<<(unsigned)((c->NT + tb - 1) / tb), tb, 0, c->stream>>>(c->inv_trace_mass, c->basis, c->g, n, c->NT);
        c->launched(2);
        const size_t tsz = c->mixed() ? sizeof(float) : sizeof(double);
        if (c->has_dg() && c->ilu2d()) {  // block ILU(0) factors instead of the block-Jacobi pool
            c->dg_perm = c->alloc<int>((size_t)c->cells * c->m);
        } else if (c->has_dg()) {
            if (c->half16()) {
                c->dg_pool = c->alloc<char>((size_t)c->cells * c->m * pad8(c->m) * sizeof(__half));
                c->dg_scale = c->alloc<float>((size_t)c->cells * c->m);
            } else {
                c->dg_pool = c->alloc<char>((size_t)c->cells * c->m * c->m * tsz);
            }
            c->dg_perm = c->alloc<int>((size_t)c->cells * c->m);
        }
        if (c->has_hdg()) {
            if (c->c32()) {  // FP32 Schur blocks and kept FP32 cell factors instead of FP64 S and X
                c->S32 = c->alloc<float>((size_t)c->cells * c->t * c->t);
                c->lu32 = c->alloc<float>((size_t)c->cells * c->m * c->m);
                c->lu32_perm = c->alloc<int>((size_t)c->cells * c->m);
                c->hq = c->alloc<double>(c->N);
            } else {
                c->S = c->alloc<double>((size_t)c->cells * c->t * c->t);
                c->X = c->alloc<double>((size_t)c->cells * c->m * c->t);
            }
            c->Y = c->alloc<double>((size_t)c->cells * c->m);
            c->cy = c->alloc<double>((size_t)c->cells * c->t);
            c->hrhs = c->alloc<double>(c->NT);
            const size_t per_cell = (size_t)c->m * (c->m + c->t + 1) * (c->c32() ? sizeof(float) : sizeof(double));
            const size_t budget = (size_t)8 << 30;  // condensation workspace: at most 8 GiB
            c->aug_cells = (int)std::max<size_t>(1, std::min<size_t>(c->cells, budget / per_cell));
            c->aug_bytes = (size_t)c->aug_cells * per_cell;
            c->aug = reinterpret_cast<double *>(c->alloc<char>(c->aug_bytes));
            if (c->c32()) c->aug32 = reinterpret_cast<float *>(c->aug);
            c->aug_perm = c->alloc<int>((size_t)c->aug_cells * c->m);
            c->face_pool = c->alloc<char>((size_t)c->faces * c->fw * c->fw * tsz);
            c->face_perm = c->alloc<int>((size_t)c->faces * c->fw);
        }
        const long long vn = std::max(c->has_dg() ? c->N : 0LL, c->has_hdg() ? c->NT : 0LL);
        c->vld = ((vn + 31) / 32) * 32;
        c->restart = k.restart;
        c->V = c->alloc<double>((size_t)c->vld * (k.restart + 1));
        c->gw = c->alloc<double>(vn);
        c->gz = c->alloc<double>(vn);
        if (c->has_dg()) {
            c->gres[DGH_OP_DG] = c->alloc<double>(c->N);
            c->gres[DGH_OP_DG_T] = c->alloc<double>(c->N);
        }
        if (c->has_hdg()) c->gres[DGH_OP_HDG] = c->alloc<double>(c->NT);
        c->gcoef = c->alloc<double>(KR_MAXK);
        c->g_rhs = c->alloc<double>(vn);
        c->g_x = c->alloc<double>(vn);
        c->gdev = c->alloc<GmresDev>(1);
        ck(cudaMemset(c->V, 0, sizeof(double) * (size_t)c->vld * (k.restart + 1)), "memset");
        if (c->has_dg() && c->mixed()) {
            if (c->overint()) {  // chunked: assembly with the over-integrated volume terms, then the LU
                const size_t per_cell = (size_t)c->m * c->m * sizeof(double);
                const size_t budget = (size_t)8 << 30;  // FP64 factor workspace: at most 8 GiB
                c->dg_ws_cells = (int)std::max<size_t>(1, std::min<size_t>(c->cells, budget / per_cell));
                c->dg_ws = c->alloc<double>((size_t)c->dg_ws_cells * c->m * c->m);
            } else {  // one persistent fused launch: an FP64 slot per resident CTA (two per SM)
                c->dg_slot_count = std::min(c->cells, 2 * c->sms);
                c->dg_slots = c->alloc<double>((size_t)c->dg_slot_count * c->m * c->m);
            }
        }
        if (c->has_dg() || c->has_hdg()) {
            const size_t smem = lu_left_smem_bytes(c->m);
            allow_dynamic_smem((const void *)k_lu_left<true>, smem);
            int per_sm = 0;
            ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lu_left<true>, LL_THREADS, smem), "occupancy");
            c->lu_grid = c->sms * std::max(1, per_sm);
            const int P = (c->m + LL_NB - 1) / LL_NB;
            c->lu_tri = c->alloc<double>((size_t)c->lu_grid * P * LL_TRI);
        }
        if (c->has_dg() && c->ilu2d()) ilu2_build(c);
        if (c->slabbed()) c->slab.buf = c->alloc<double>(16);
        c->sync();
    });
    if (rc != DGH_OK) {
        g_create_error = c->err;
        dgh_ctx_destroy(c);
        return rc;
    }
    *out = c;
    return DGH_OK;
}
}  // namespace

extern "C" {

int dgh_ctx_destroy(dgh_ctx *c) {
    if (!c) return DGH_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto &r : c->pending) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (auto e : c->spare) cudaEventDestroy(e);
    for (void *p : c->owned) cudaFree(p);
    if (c->pinned) cudaFreeHost(c->pinned);
    for (auto &g : c->cycle)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    if (c->ilu2.blas) cublasDestroy(c->ilu2.blas);
    if (c->aux) cudaStreamDestroy(c->aux);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return DGH_OK;
}

const char *dgh_last_error(const dgh_ctx *c) { return c ? c->err.c_str() : g_create_error.c_str(); }

int dgh_sizes(const dgh_ctx *c, int64_t s[8]) {
    if (!c || !s) return DGH_ERR_INVALID;
    s[0] = c->N; s[1] = c->NT; s[2] = c->m; s[3] = c->cells; s[4] = c->faces; s[5] = c->n; s[6] = c->t; s[7] = c->fw;
    return DGH_OK;
}
void *dgh_stream(const dgh_ctx *c) { return c ? (void *)c->stream : nullptr; }
int dgh_get_config(const dgh_ctx *c, dgh_config *out) {
    if (!c || !out) return DGH_ERR_INVALID;
    *out = c->cfg;
    return DGH_OK;
}
int dgh_geometry(const dgh_ctx *c, double out[4]) {
    if (!c || !out) return DGH_ERR_INVALID;
    out[0] = c->g.hx; out[1] = c->g.hy; out[2] = c->cs.lx; out[3] = c->cs.ly;  // 1D: h, 1, 2, 1
    return DGH_OK;
}
int dgh_nodes(const dgh_ctx *c, double *x, double *w) {
    if (!c) return DGH_ERR_INVALID;
    for (int i = 0; i < c->n; ++i) {
        if (x) x[i] = c->xnodes[i];
        if (w) w[i] = c->basis.w[i];
    }
    return DGH_OK;
}
int dgh_sync(dgh_ctx *c) { return guard(c, [&] { c->sync(); }); }
int dgh_device_bytes(const dgh_ctx *c, int64_t *b) {
    if (!c || !b) return DGH_ERR_INVALID;
    *b = (int64_t)c->bytes;
    return DGH_OK;
}
int64_t dgh_launch_count(const dgh_ctx *c) { return c ? c->launches : 0; }
int dgh_timing_enable(dgh_ctx *c, int on) {
    return guard(c, [&] {
        c->flush_timers();
        for (int k = 0; k < DGH_TIMER_COUNT; ++k) {
            c->t_ms[k] = 0;
            c->t_n[k] = 0;
        }
        c->timing = on != 0;
    });
}
int dgh_timing_read(dgh_ctx *c, int category, double *ms, int64_t *count) {
    return guard(c, [&] {
        need(category >= 0 && category < DGH_TIMER_COUNT, "Invalid timer category");
        c->flush_timers();
        if (ms) *ms = c->t_ms[category];
        if (count) *count = c->t_n[category];
    });
}

int dgh_vec_alloc(dgh_ctx *c, int64_t n, double **dev) {
    return guard(c, [&] {
        need(dev && n > 0, "Invalid vector size");
        ck(cudaMalloc((void **)dev, n * sizeof(double)), "cudaMalloc");
        ck(cudaMemsetAsync(*dev, 0, n * sizeof(double), c->stream), "memset");
    });
}
int dgh_vec_free(dgh_ctx *c, double *dev) {
    return guard(c, [&] { ck(cudaFree(dev), "cudaFree"); });
}
int dgh_upload(dgh_ctx *c, double *dev, const double *host, int64_t n) {
    return guard(c, [&] { ck(cudaMemcpyAsync(dev, host, n * sizeof(double), cudaMemcpyHostToDevice, c->stream), "h2d"); });
}
int dgh_download(dgh_ctx *c, double *host, const double *dev, int64_t n) {
    return guard(c, [&] {
        ck(cudaMemcpyAsync(host, dev, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "d2h");
        c->sync();
    });
}
int dgh_axpby(dgh_ctx *c, double a, const double *x, double b, const double *y, double *out, int64_t n) {
    return guard(c, [&] { axpby(c, a, x, b, y, out, n); });
}

// ---- Problem ------------------------------------------------------------------------------------
int dgh_initial(dgh_ctx *c, double *u) {
    return guard(c, [&] {
        need(u, "null state");
        if (c->d1()) {
            DGH_DISPATCH_N(c->n, {
                k1_initial<N><<<grid1(c->cells, 64), 64, 0, c->stream>>>(u, c->rule, c->b1, c->g1, c->cs, c->status);
            });
        } else {
            // a slab projects its interior cells, at their global rows, then fills its ghost rows
            int first = 0, count = 0;
            interior_cells(c, first, count);
            Grid gi = c->g;
            gi.row0 = c->slabbed() ? c->slab.row0 : 0;
            double *ui = u + (size_t)first * c->m;
            DGH_DISPATCH_N(c->n, { k_initial<N><<<count, 256, 0, c->stream>>>(ui, c->rule, c->basis, gi, c->cs, c->status); });
        }
        c->launched();
        c->check_status();
        slab_halo(c, u);
        // initial_and_error.cpp:53 — the projected state must be admissible
        const int one = 1;
        std::memcpy(c->pinned, &one, sizeof(int));
        ck(cudaMemcpyAsync(c->ok, c->pinned, sizeof(int), cudaMemcpyHostToDevice, c->stream), "copy");
        launch_trace(c, u, c->traces, true);
        ck(cudaMemcpyAsync(c->pinned, c->ok, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "copy");
        c->sync();
        int ok = 0;
        std::memcpy(&ok, c->pinned, sizeof(int));
        if (c->slabbed()) {
            double bad = ok ? 0. : 1.;
            c->slab_reduce(&bad, 1, 1);
            ok = bad > 0 ? 0 : 1;
        }
        if (!ok) fail(DGH_ERR_STATE, "Invalid projected initial state");
    });
}

int dgh_freeze(dgh_ctx *c, const double *u, double *rate) {
    return guard(c, [&] {
        need(u && rate, "null argument");
        slab_halo(c, u);
        ck(cudaMemcpyAsync(c->old, u, c->N * sizeof(double), cudaMemcpyDeviceToDevice, c->stream), "copy");
        launch_trace(c, u, c->traces, false);
        if (c->d1()) {
            // dg_hdg_1d/src/discretization.cpp:75-92
            const unsigned nb = grid1(c->cells, 256);
            k1_speeds<<<grid1(c->cells), K1_THREADS, 0, c->stream>>>(c->traces, c->speeds, c->g1, c->cfg.safety,
                                                                     c->status);
            DGH_DISPATCH_N(c->n, { k1_rate<N><<<nb, 256, 0, c->stream>>>(u, c->speeds, c->partial, c->b1, c->g1); });
            c->launched(2);
            c->check_status();
            std::vector<double> part(nb);
            ck(cudaMemcpyAsync(part.data(), c->partial, nb * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "copy");
            c->sync();
            double r = 0;
            for (double p : part) r = r < p ? p : r;
            if (!(std::isfinite(r) && r > 0)) fail(DGH_ERR_STATE, "Invalid CFL rate");
            *rate = r;
            c->frozen = true;
            c->linearised = c->dg_factored = c->condensed = c->face_factored = false;
            return;
        }
        int first = 0, count = 0;  // the rate of a slab is the maximum over its interior cells
        interior_cells(c, first, count);
        DGH_DISPATCH_N(c->n, {
            const int tot = 2 * c->cells * N;
            k_speeds<N><<<(tot + 255) / 256, 256, 0, c->stream>>>(c->traces, c->speeds, c->g, c->cfg.safety, c->status);
            using T = Team<N>;
            if (c->overint())
                k_rate_q<N><<<std::min(c->cells, c->sms * 4), Q_THREADS, 0, c->stream>>>(u, c->speeds, c->bq, c->g, c->partial, c->status);
            else
                k_rate<N><<<(count + T::CPB - 1) / T::CPB, T::THREADS, 0, c->stream>>>(u, c->speeds, c->g, c->partial,
                                                                                     c->status, first, first + count);
        });
        c->launched(2);
        c->check_status();
        DGH_DISPATCH_N(c->n, {
            const int nb = c->overint() ? std::min(c->cells, c->sms * 4) : (count + Team<N>::CPB - 1) / Team<N>::CPB;
            std::vector<double> part(nb);
            ck(cudaMemcpyAsync(part.data(), c->partial, nb * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "copy");
            c->sync();
            double r = 0;
            for (double p : part) r = std::max(r, p);
            c->slab_reduce(&r, 1, 1);
            *rate = r;
        });
        c->frozen = true;
        c->linearised = c->dg_factored = c->condensed = c->face_factored = false;
    });
}

int dgh_set_stage(dgh_ctx *c, const double *old, double step) {
    return guard(c, [&] {
        need(old, "null argument");
        if (old != c->old)
            ck(cudaMemcpyAsync(c->old, old, c->N * sizeof(double), cudaMemcpyDeviceToDevice, c->stream), "copy");
        c->step_size = step;
        c->inv_step = 1. / step;
        c->linearised = c->dg_factored = c->condensed = c->face_factored = false;
    });
}

int dgh_residual(dgh_ctx *c, const double *u, double *r) {
    return guard(c, [&] {
        need(u && r, "null argument");
        need(c->frozen, "Freeze the wave speeds before evaluating the residual");
        Timed tm(c, DGH_TIMER_RESIDUAL);
        slab_halo(c, u);
        launch_trace(c, u, c->traces, false);
        if (c->d1()) {
            DGH_DISPATCH_N(c->n, {
                k1_residual<N><<<grid1(c->cells), K1_THREADS, 0, c->stream>>>(u, c->old, c->traces, c->speeds, r, c->b1,
                                                                              c->g1, 1. / c->step_size);
            });
            c->launched();
            return;
        }
        DGH_DISPATCH_N(c->n, {
            using T = Team<N>;
            k_residual<N><<<c->team_blocks(T::CPB), T::THREADS, 0, c->stream>>>(u, c->old, c->traces, c->speeds, r,
                                                                               c->basis, c->g, 1. / c->step_size,
                                                                               c->overint() ? 0 : 1);
            if (c->overint()) {
                k_vol_residual_q<N><<<std::min(c->cells, c->sms * 4), Q_THREADS, 0, c->stream>>>(u, r, c->bq, c->g);
                c->launched();
            }
        });
        c->launched();
        slab_zero_ghosts(c, r);
    });
}

int dgh_admissible(dgh_ctx *c, const double *u, int *okp) {
    return guard(c, [&] {
        need(u && okp, "null argument");
        slab_halo(c, u);  // ghost cells are the neighbours' cells: checking them changes nothing
        const int one = 1;
        std::memcpy(c->pinned, &one, sizeof(int));
        ck(cudaMemcpyAsync(c->ok, c->pinned, sizeof(int), cudaMemcpyHostToDevice, c->stream), "copy");
        launch_trace(c, u, c->traces, true);
        ck(cudaMemcpyAsync(c->pinned, c->ok, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "copy");
        c->sync();
        std::memcpy(okp, c->pinned, sizeof(int));
        if (c->slabbed()) {  // admissible on every slab
            double bad = *okp ? 0. : 1.;
            c->slab_reduce(&bad, 1, 1);
            *okp = bad > 0 ? 0 : 1;
        }
    });
}

int dgh_trace(dgh_ctx *c, const double *u, double *lam) {
    return guard(c, [&] {
        need(c->frozen, "Freeze the wave speeds first");
        slab_halo(c, u);
        launch_trace(c, u, c->traces, false);
        if (c->d1()) {
            k1_trace_lambda<<<grid1(c->cells), K1_THREADS, 0, c->stream>>>(c->traces, c->speeds, lam, c->g1);
            c->launched();
            return;
        }
        DGH_DISPATCH_N(c->n, {
            const int tot = 2 * c->cells * N;
            k_trace_lambda<N><<<(tot + 255) / 256, 256, 0, c->stream>>>(c->traces, c->speeds, lam, c->g);
        });
        c->launched();
        slab_zero_ghost_faces(c, lam);
    });
}

int dgh_dual_norm(dgh_ctx *c, const double *r, double *out) {
    return guard(c, [&] { *out = std::sqrt(c->reduce_scalar(r, c->mass, true, c->N, true)); });
}
int dgh_state_norm(dgh_ctx *c, const double *u, double *out) {
    return guard(c, [&] { *out = std::sqrt(c->reduce_scalar(u, c->mass, false, c->N, true)); });
}

int dgh_integral(dgh_ctx *c, const double *u, double out[4]) {
    return guard(c, [&] {
        if (c->d1()) {
            DGH_DISPATCH_N(c->n, { k1_integral<N><<<grid1(c->cells), K1_THREADS, 0, c->stream>>>(u, c->b1, c->g1, c->partial); });
        } else {
            DGH_DISPATCH_N(c->n, {
                const int tot = c->cells * NVAR;
                k_integral<N><<<(tot + 255) / 256, 256, 0, c->stream>>>(u, c->basis, c->g, c->partial);
            });
        }
        c->launched();
        std::vector<double> part((size_t)c->cells * 4);
        ck(cudaMemcpyAsync(part.data(), c->partial, part.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "copy");
        c->sync();
        int first = 0, count = 0;
        interior_cells(c, first, count);
        for (int v = 0; v < 4; ++v) out[v] = 0;
        for (int cell = first; cell < first + count; ++cell)
            for (int v = 0; v < 4; ++v) out[v] += part[(size_t)cell * 4 + v];
        c->slab_reduce(out, 4, 0);
    });
}

int dgh_l2_error(dgh_ctx *c, const double *u, double time, double out[4]) {
    return guard(c, [&] {
        if (c->d1()) {
            DGH_DISPATCH_N(c->n, {
                k1_l2_error<N><<<grid1(c->cells), K1_THREADS, 0, c->stream>>>(u, c->rule, c->g1, c->cs, time, c->partial,
                                                                              c->status);
            });
        } else {
            int first = 0, count = 0;  // a slab: its interior cells at their global rows
            interior_cells(c, first, count);
            Grid gi = c->g;
            gi.row0 = c->slabbed() ? c->slab.row0 : 0;
            DGH_DISPATCH_N(c->n, {
                k_l2_error<N><<<count, 256, 0, c->stream>>>(u + (size_t)first * c->m, c->rule, c->basis, gi, c->cs, time,
                                                            c->partial, c->status);
            });
        }
        c->launched();
        c->check_status();
        const int cells = c->slabbed() ? c->g.nx * c->slab.rows : c->cells;
        std::vector<double> part((size_t)cells * 4);
        ck(cudaMemcpyAsync(part.data(), c->partial, part.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "copy");
        c->sync();
        for (int v = 0; v < 4; ++v) out[v] = 0;
        for (int cell = 0; cell < cells; ++cell)
            for (int v = 0; v < 4; ++v) out[v] += part[(size_t)cell * 4 + v];
        c->slab_reduce(out, 4, 0);
        for (int v = 0; v < 4; ++v) out[v] = std::sqrt(out[v]);
    });
}

int dgh_copy_speeds(dgh_ctx *c, double *dev_ab) {
    return guard(c, [&] {
        need(c->frozen, "Freeze the wave speeds first");
        ck(cudaMemcpyAsync(dev_ab, c->speeds, c->nspeeds * sizeof(double), cudaMemcpyDeviceToDevice,
                           c->stream), "copy");
    });
}
int dgh_set_speeds(dgh_ctx *c, const double *dev_ab) {
    return guard(c, [&] {
        ck(cudaMemcpyAsync(c->speeds, dev_ab, c->nspeeds * sizeof(double), cudaMemcpyDeviceToDevice,
                           c->stream), "copy");
        c->frozen = true;
        c->linearised = c->dg_factored = c->condensed = c->face_factored = false;
    });
}
int dgh_mass_axpby(dgh_ctx *c, double a, const double *x, double b, const double *y, double *out) {
    return guard(c, [&] {
        k_mass_axpby<<<c->red_grid, KR_THREADS, 0, c->stream>>>(a, x, c->mass, b, y, out, c->N);
        c->launched();
    });
}
int dgh_rho2(dgh_ctx *c, const double *u, double *value, double *grad) {
    return guard(c, [&] {
        need(!c->d1(), "The adjoint objective is built for the 2D problem only");
        need(!c->slabbed(), "The adjoint objective is not built for slab contexts");
        k_rho2<<<c->red_grid, KR_THREADS, 0, c->stream>>>(u, c->mass, c->P, c->N, grad, c->partial);
        k_reduce<<<1, KR_THREADS, 0, c->stream>>>(c->partial, c->red_grid, c->red);
        c->launched(2);
        ck(cudaMemcpyAsync(c->pinned, c->red, sizeof(double), cudaMemcpyDeviceToHost, c->stream), "copy");
        c->sync();
        *value = c->pinned[0];
    });
}
int dgh_speeds(dgh_ctx *c, double *host_ab) {
    return guard(c, [&] {
        ck(cudaMemcpyAsync(host_ab, c->speeds, c->nspeeds * sizeof(double), cudaMemcpyDeviceToHost,
                           c->stream), "copy");
        c->sync();
    });
}

// ---- DGOperator --------------------------------------------------------------------------------
namespace {
void linearise(dgh_ctx *c, const double *u) {
    need(c->frozen, "Freeze the wave speeds before refreshing the Jacobian");
    need(c->step_size > 0, "Set the time step before refreshing the Jacobian");
    slab_halo(c, u);
    launch_trace(c, u, c->traces, false);
    if (c->d1()) {
        DGH_DISPATCH_N(c->n, {
            k1_linearise<N><<<grid1(c->cells), K1_THREADS, 0, c->stream>>>(u, c->traces, c->speeds, c->vol, c->fcache,
                                                                           c->b1, c->g1);
        });
        c->launched();
        c->linearised = true;
        c->dg_factored = c->condensed = c->face_factored = false;
        return;
    }
    DGH_DISPATCH_N(c->n, {
        const long long tv = (long long)c->cells * N * N;
        k_volume_cache<N><<<(unsigned)((tv + 255) / 256), 256, 0, c->stream>>>(u, c->vol, c->g);
        if (c->overint()) {
            k_volume_cache_q<N><<<std::min(c->cells, c->sms * 4), Q_THREADS, 0, c->stream>>>(u, c->volq, c->bq, c->g);
            c->launched();
        }
        const int tf = 2 * c->cells * N;
        k_face_cache<N><<<(tf + 255) / 256, 256, 0, c->stream>>>(c->traces, c->speeds, c->fcache, c->basis, c->g);
    });
    c->launched(2);
    c->linearised = true;
    c->dg_factored = c->condensed = c->face_factored = false;
}
}  // namespace

int dgh_dg_refresh(dgh_ctx *c, const double *u) {
    return guard(c, [&] { linearise(c, u); });
}
int dgh_dg_apply(dgh_ctx *c, const double *v, double *jv) {
    return guard(c, [&] { dg_apply(c, v, jv); });
}
int dgh_dg_apply_T(dgh_ctx *c, const double *w, double *jtw) {
    return guard(c, [&] { dg_apply_t(c, w, jtw); });
}
int dgh_dg_block(dgh_ctx *c, int row, int col, double *host_block) {
    return guard(c, [&] {
        need(c->linearised, "Refresh the volume Jacobian before assembling a block");
        need(row >= 0 && row < c->cells && col >= 0 && col < c->cells, "Invalid block index");
        int side = -1;
        if (row != col && !c->d1())
            for (int sd = 0; sd < 4; ++sd)
                if (neighbor(c->g, row, sd) == col) side = sd;
        need(row == col || side >= 0, "Only diagonal and face-neighbour cell blocks exist on the device");
        double *tmp = c->alloc<double>((size_t)c->m * c->m);
        if (side >= 0) {  // coupling block (dg_operator.cpp:22-48, col != row)
            double **dst = c->alloc<double *>(1);
            int *pair = c->alloc<int>(2);
            const int hp[2] = {row, side};
            ck(cudaMemcpy(dst, &tmp, sizeof(double *), cudaMemcpyHostToDevice), "copy");
            ck(cudaMemcpy(pair, hp, sizeof hp, cudaMemcpyHostToDevice), "copy");
            DGH_DISPATCH_N(c->n, {
                k_dg_coupling<N, double><<<1, 256, 0, c->stream>>>(dst, pair, 1, c->fcache, c->speeds, c->basis, c->g);
            });
            c->sync();
            for (void *q : {(void *)pair, (void *)dst}) {  // the two small allocations, newest first
                ck(cudaFree(q), "cudaFree");
                c->owned.pop_back();
                c->bytes -= 16;
            }
        } else if (c->d1()) {
            DGH_DISPATCH_N(c->n, {
                k1_dg_assemble<N, double><<<grid1((long long)c->m * c->m), K1_THREADS, 0, c->stream>>>(
                    tmp, c->vol, c->fcache, c->b1, c->g1, c->inv_step, row, 1);
            });
        } else {
            DGH_DISPATCH_N(c->n, {
                k_dg_assemble<N, double><<<1, 256, 0, c->stream>>>(tmp, c->vol, c->fcache, c->speeds, c->basis, c->g,
                                                                    c->inv_step, row, 1, c->overint() ? 0 : 1);
                if (c->overint()) {
                    k_vol_block_q<N, double><<<1, Q_THREADS, 0, c->stream>>>(tmp, c->m, c->volq, c->bq, c->g, row, 1);
                    c->launched();
                }
            });
        }
        c->launched();
        ck(cudaMemcpyAsync(host_block, tmp, (size_t)c->m * c->m * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "copy");
        c->sync();
        ck(cudaFree(tmp), "cudaFree");
        c->owned.pop_back();
        c->bytes -= std::max<size_t>((size_t)c->m * c->m * sizeof(double), 16);
    });
}

}  // extern "C"

// ---- factorisation variants and the per-degree autotuner ------------------------------------------
namespace {
std::mutex g_tune_mutex;
std::map<std::tuple<int, int, int, int>, int> g_tune_cache;  // (kind, n, precision, cells of kind 3) -> variant

// DG blocks of cells [first, first + count): assembly and LU with the given variant.
void dg_factor(dgh_ctx *c, int variant, int first, int count) {
    const size_t stride = (size_t)c->m * c->m;
    const int grid = std::min(count, c->sms * 8);
    if (c->mixed() && (c->half16() || variant == 0) && !c->overint()) {
        // one persistent launch: assemble + FP64 left-looking LU per CTA slot, reduced output
        DGH_DISPATCH_N(c->n, { launch_dg_fused<N>(c, first, count); });
        return;
    }
    if (c->half16()) {  // FP64 left-looking in the workspace, then FP16 slabs with row scales
        const int mp = pad8(c->m);
        for (int f = first; f < first + count; f += c->dg_ws_cells) {
            const int cnt = std::min(c->dg_ws_cells, first + count - f);
            DGH_DISPATCH_N(c->n, {
                k_dg_assemble<N, double><<<std::min(cnt, c->sms * 8), 256, 0, c->stream>>>(
                    c->dg_ws, c->vol, c->fcache, c->speeds, c->basis, c->g, c->inv_step, f, cnt, c->overint() ? 0 : 1);
                if (c->overint()) {
                    k_vol_block_q<N, double><<<std::min(cnt, c->sms * 4), Q_THREADS, 0, c->stream>>>(
                        c->dg_ws, c->m, c->volq, c->bq, c->g, f, cnt);
                    c->launched();
                }
            });
            c->launched();
            launch_lu_left<false>(c, c->dg_ws, stride, c->m, c->m, cnt, c->dg_perm + (size_t)f * c->m, ST_SINGULAR, false);
            const long long warps = (long long)cnt * ((c->m + 31) / 32);
            k_pack_half<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, c->stream>>>(
                c->dg_ws, c->m, cnt, (__half *)c->dg_pool + (size_t)f * c->m * mp, c->dg_scale + (size_t)f * c->m);
            c->launched();
        }
        return;
    }
    if (c->mixed()) {
        if (variant == 0) {  // FP64 left-looking in the workspace, FP32 slabs out, chunked
            for (int f = first; f < first + count; f += c->dg_ws_cells) {
                const int cnt = std::min(c->dg_ws_cells, first + count - f);
                DGH_DISPATCH_N(c->n, {
                    k_dg_assemble<N, double><<<std::min(cnt, c->sms * 8), 256, 0, c->stream>>>(
                        c->dg_ws, c->vol, c->fcache, c->speeds, c->basis, c->g, c->inv_step, f, cnt, c->overint() ? 0 : 1);
                    if (c->overint()) {
                        k_vol_block_q<N, double><<<std::min(cnt, c->sms * 4), Q_THREADS, 0, c->stream>>>(
                            c->dg_ws, c->m, c->volq, c->bq, c->g, f, cnt);
                        c->launched();
                    }
                });
                c->launched();
                launch_lu_left<false>(c, c->dg_ws, stride, c->m, c->m, cnt, c->dg_perm + (size_t)f * c->m, ST_SINGULAR,
                                      false, (float *)c->dg_pool + (size_t)f * stride);
            }
        } else {  // FP32 right-looking in place
            float *pool = (float *)c->dg_pool + (size_t)first * stride;
            DGH_DISPATCH_N(c->n, {
                k_dg_assemble<N, float><<<grid, 256, 0, c->stream>>>(pool, c->vol, c->fcache, c->speeds, c->basis, c->g,
                                                                     c->inv_step, first, count, c->overint() ? 0 : 1);
                if (c->overint()) {
                    k_vol_block_q<N, float><<<std::min(count, c->sms * 4), Q_THREADS, 0, c->stream>>>(
                        pool, c->m, c->volq, c->bq, c->g, first, count);
                    c->launched();
                }
            });
            c->launched();
            launch_lu<float>(c, pool, stride, c->m, c->m, count, c->dg_perm + (size_t)first * c->m, ST_SINGULAR, true);
        }
    } else {
        double *pool = (double *)c->dg_pool + (size_t)first * stride;
        DGH_DISPATCH_N(c->n, {
            k_dg_assemble<N, double><<<grid, 256, 0, c->stream>>>(pool, c->vol, c->fcache, c->speeds, c->basis, c->g,
                                                                  c->inv_step, first, count, c->overint() ? 0 : 1);
            if (c->overint()) {
                k_vol_block_q<N, double><<<std::min(count, c->sms * 4), Q_THREADS, 0, c->stream>>>(
                    pool, c->m, c->volq, c->bq, c->g, first, count);
                c->launched();
            }
        });
        c->launched();
        if (variant == 0)
            launch_lu_left<false>(c, pool, stride, c->m, c->m, count, c->dg_perm + (size_t)first * c->m, ST_SINGULAR, true);
        else
            launch_lu<double>(c, pool, stride, c->m, c->m, count, c->dg_perm + (size_t)first * c->m, ST_SINGULAR, true);
    }
}
// Condensation of cells [first, first + count) (count <= aug_cells): [A | B | r], LU + solve
// with the given variant, S, X, y, C y.
void hdg_condense_chunk(dgh_ctx *c, int variant, const double *r, int first, int count) {
    const int ld = c->m + c->t + 1, grid = std::min(count, c->sms * 8);
    DGH_DISPATCH_N(c->n, {
        k_hdg_assemble<N, double><<<grid, 256, 0, c->stream>>>(c->aug, c->vol, c->fcache, c->speeds, r, c->basis, c->g,
                                                               c->inv_step, first, count, c->overint() ? 0 : 1);
        if (c->overint()) {
            k_vol_block_q<N, double><<<std::min(count, c->sms * 4), Q_THREADS, 0, c->stream>>>(
                c->aug, ld, c->volq, c->bq, c->g, first, count);
            c->launched();
        }
    });
    c->launched();
    if (variant == 0) {  // X and y straight to their persistent arrays
        launch_lu_left<true>(c, c->aug, (size_t)c->m * ld, c->m, ld, count, c->aug_perm, ST_SINGULAR_HDG, false, nullptr,
                             c->X + (size_t)first * c->m * c->t, c->Y + (size_t)first * c->m);
    } else {
        launch_lu<double>(c, c->aug, (size_t)c->m * ld, c->m, ld, count, c->aug_perm, ST_SINGULAR_HDG, false);
        constexpr size_t bs_smem = backsolve_smem_bytes();
        allow_dynamic_smem((const void *)k_backsolve_dmma, bs_smem);
        int per_sm = 0;
        ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_backsolve_dmma, LU_THREADS, bs_smem), "occupancy");
        k_backsolve_dmma<<<std::min(count, c->sms * std::max(1, per_sm)), LU_THREADS, bs_smem, c->stream>>>(
            c->aug, (size_t)c->m * ld, c->m, ld, count);
        c->launched();
    }
    DGH_DISPATCH_N(c->n, {
        if (variant == 0)
            k_hdg_schur<N, double, true><<<grid, 256, 0, c->stream>>>(c->aug, c->fcache, c->speeds, c->S, c->X, c->Y,
                                                                      c->cy, c->basis, c->g, first, count);
        else
            k_hdg_schur<N, double, false><<<grid, 256, 0, c->stream>>>(c->aug, c->fcache, c->speeds, c->S, c->X, c->Y,
                                                                       c->cy, c->basis, c->g, first, count);
    });
    c->launched();
}
// Cells per chunk of the condensation workspace for augmented matrices of element type T.
template <typename T> int aug_chunk(const dgh_ctx *c) {
    return (int)std::max<size_t>(1, std::min<size_t>(c->cells, c->aug_bytes / ((size_t)c->m * (c->m + c->t + 1) *
                                                                                 sizeof(T))));
}
// FP32-storage condensation of cells [first, first + count), variant 0: [A | B | r] assembled in
// FP64, the left-looking LU on the FP64 tensor pipe with the fused right-hand-side solve, the
// factors rounded into the cells' FP32 slabs, then S = -C X stored in FP32, y and C y in FP64.
void hdg_condense_chunk32_tc(dgh_ctx *c, const double *r, int first, int count) {
    const int ld = c->m + c->t + 1, grid = std::min(count, c->sms * 8);
    const size_t stride = (size_t)c->m * ld;
    DGH_DISPATCH_N(c->n, {
        k_hdg_assemble<N, double><<<grid, 256, 0, c->stream>>>(c->aug, c->vol, c->fcache, c->speeds, r, c->basis, c->g,
                                                               c->inv_step, first, count, c->overint() ? 0 : 1);
        if (c->overint()) {
            k_vol_block_q<N, double><<<std::min(count, c->sms * 4), Q_THREADS, 0, c->stream>>>(
                c->aug, ld, c->volq, c->bq, c->g, first, count);
            c->launched();
        }
    });
    c->launched();
    int *perm = c->lu32_perm + (size_t)first * c->m;
    launch_lu_left<true>(c, c->aug, stride, c->m, ld, count, perm, ST_SINGULAR_HDG, false);
    const long long warps = (long long)count * ((c->m + 31) / 32);
    k_slab_pack<double, float><<<(unsigned)((warps * 32 + 255) / 256), 256, 0, c->stream>>>(
        c->aug, stride, c->m, ld, count, c->lu32 + (size_t)first * c->m * c->m, perm);
    c->launched();
    DGH_DISPATCH_N(c->n, {
        k_hdg_schur<N, double, false, float><<<grid, 256, 0, c->stream>>>(c->aug, c->fcache, c->speeds, c->S32, nullptr,
                                                                          c->Y, c->cy, c->basis, c->g, first, count);
    });
    c->launched();
}
// Variant 1: [A | B | r] assembled in FP32, right-looking FP32 LU with FP32 accumulation (the L
// fix-up kept), the factors copied to the cells' FP32 slabs for later solves, back substitution
// for X | y, then S = -C X stored in FP32, y and C y in FP64.
void hdg_condense_chunk32(dgh_ctx *c, const double *r, int first, int count) {
    const int ld = c->m + c->t + 1, grid = std::min(count, c->sms * 8);
    const size_t stride = (size_t)c->m * ld;
    DGH_DISPATCH_N(c->n, {
        k_hdg_assemble<N, float><<<grid, 256, 0, c->stream>>>(c->aug32, c->vol, c->fcache, c->speeds, r, c->basis, c->g,
                                                              c->inv_step, first, count, c->overint() ? 0 : 1);
        if (c->overint()) {
            k_vol_block_q<N, float><<<std::min(count, c->sms * 4), Q_THREADS, 0, c->stream>>>(
                c->aug32, ld, c->volq, c->bq, c->g, first, count);
            c->launched();
        }
    });
    c->launched();
    launch_lu<float>(c, c->aug32, stride, c->m, ld, count, c->lu32_perm + (size_t)first * c->m, ST_SINGULAR_HDG, false,
                     true);
    const long long warps = (long long)count * ((c->m + 31) / 32);
    k_slab_pack<float, float><<<(unsigned)((warps * 32 + 255) / 256), 256, 0, c->stream>>>(
        c->aug32, stride, c->m, ld, count, c->lu32 + (size_t)first * c->m * c->m);
    k_backsolve<float><<<std::min(count, c->sms * 8), LU_THREADS, 0, c->stream>>>(c->aug32, stride, c->m, ld, count);
    c->launched(2);
    DGH_DISPATCH_N(c->n, {
        k_hdg_schur<N, float, false, float><<<grid, 256, 0, c->stream>>>(c->aug32, c->fcache, c->speeds, c->S32, nullptr,
                                                                         c->Y, c->cy, c->basis, c->g, first, count);
    });
    c->launched();
}
// Condensed right-hand side from the cells' C y (g = 0 on the projected trace).
void hdg_rhs_from_cy(dgh_ctx *c) {
    DGH_DISPATCH_N(c->n, {
        const long long tot = c->NT;
        k_hdg_rhs<N><<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(c->cy, c->hrhs, c->g);
    });
    c->launched();
}
// Times f(variant) for variants 0 and 1 (best of two runs each) and returns the faster one.
template <class F> int tune_pick(dgh_ctx *c, F &&f, double *ms_out) {
    cudaEvent_t a = c->event(), b = c->event();
    double best[2] = {1e300, 1e300};
    for (int rep = 0; rep < 2; ++rep)
        for (int v = 0; v < 2; ++v) {
            ck(cudaEventRecord(a, c->stream), "cudaEventRecord");
            f(v);
            ck(cudaEventRecord(b, c->stream), "cudaEventRecord");
            ck(cudaEventSynchronize(b), "cudaEventSynchronize");
            float ms = 0;
            ck(cudaEventElapsedTime(&ms, a, b), "cudaEventElapsedTime");
            best[v] = std::min(best[v], (double)ms);
        }
    c->spare.push_back(a);
    c->spare.push_back(b);
    ms_out[0] = best[0];
    ms_out[1] = best[1];
    return best[1] < best[0] ? 1 : 0;
}
// The cached or newly tuned variant of one kind (0 DG blocks, 1 FP64 condensation, 2 FP32-storage
// condensation, 3 the DG block solve's grid shape, which also depends on the block count, 4 the
// fused DG factorisation's CTAs per SM, variant v = v + 1 CTAs).
template <class F> int tuned_variant(dgh_ctx *c, int kind, F &&time_both, double *ms_out) {
    if (!c->cfg.autotune) return 0;
    const auto key = std::make_tuple(kind, c->n, c->cfg.precision, kind == 3 ? c->cells : 0);
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) return it->second;
    }
    int v = tune_pick(c, time_both, ms_out);
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tune_cache[key] = v;
    }
    return v;
}
// The same, agreed over the ranks of a slab context (the larger variant wins), so that every
// rank factors alike and takes the same collective steps afterwards.
template <class F> int tuned_variant_all(dgh_ctx *c, int kind, F &&time_both, double *ms_out) {
    int v = tuned_variant(c, kind, time_both, ms_out);
    if (c->slabbed() && c->cfg.autotune) {
        double d = v;
        c->slab_reduce(&d, 1, 1);
        v = (int)d;
    }
    return v;
}
}  // namespace

extern "C" {

// ---- BlockJacobi -------------------------------------------------------------------------------
int dgh_block_jacobi_refresh(dgh_ctx *c, int op) {
    return guard(c, [&] {
        Timed tm(c, op == DGH_OP_DG ? DGH_TIMER_FACTOR : DGH_TIMER_FACE_FACTOR);
        if (c->d1()) {
            // BlockPreconditioner of the block-Jacobi kind (common/src/linalg/block_ilu.cpp:48-61): the
            // DenseLU of every diagonal block, whose require() texts report a failure.
            const bool dg = op == DGH_OP_DG;
            need(dg ? c->dg_pool != nullptr : c->face_pool != nullptr,
                 dg ? "context has no DG operator" : "context has no HDG operator");
            need(dg ? c->linearised : c->condensed, dg ? "Refresh the volume Jacobian before assembling a block"
                                                       : "Condense the HDG operator before refreshing its preconditioner");
            const long long tot = dg ? (long long)c->cells * c->m * c->m : (long long)c->cells * 9;
            if (c->ilu()) {
                // BlockPreconditioner::refresh (block_ilu.hpp:14-19): every pattern block, then
                // the sequential ILU(0) factorisation
                auto &pl = dg ? c->ilu_dg : c->ilu_hdg;
                const long long nb = (long long)pl.nnz * pl.m * pl.m;
                auto run = [&](auto *vals) {
                    using TF = std::remove_pointer_t<decltype(vals)>;
                    if (dg) DGH_DISPATCH_N(c->n, {
                            k1_ilu_dg_blocks<N, TF><<<grid1(nb), K1_THREADS, 0, c->stream>>>(
                                vals, pl.slot_row, pl.col, pl.nnz, c->vol, c->fcache, c->b1, c->g1, c->inv_step);
                        })
                    else k1_ilu_face_blocks<TF><<<grid1(nb), K1_THREADS, 0, c->stream>>>(vals, pl.slot_row, pl.col, pl.nnz,
                                                                                         c->S, c->speeds, c->g1);
                    k1_ilu_factor<TF><<<1, ILU_THREADS, 0, c->stream>>>(vals, pl.perm, pl.row_ptr, pl.col, pl.diag,
                                                                        pl.upd_off, pl.upd_target, pl.upd_upper, pl.rows,
                                                                        pl.m, c->status);
                    c->launched(2);
                };
                if (c->mixed()) run((float *)pl.vals);
                else run((double *)pl.vals);
                c->check_status();
                (dg ? c->dg_factored : c->face_factored) = true;
                return;
            }
            if (c->mixed()) {
                if (dg) DGH_DISPATCH_N(c->n, {
                        k1_dg_assemble<N, float><<<grid1(tot), K1_THREADS, 0, c->stream>>>(
                            (float *)c->dg_pool, c->vol, c->fcache, c->b1, c->g1, c->inv_step, 0, c->cells);
                    })
                else k1_face_blocks<float><<<grid1(tot), K1_THREADS, 0, c->stream>>>(c->S, c->speeds, (float *)c->face_pool, c->g1);
                c->launched();
                if (dg) launch_small_lu<float>(c, (float *)c->dg_pool, (size_t)c->m * c->m, c->m, c->m, c->cells, c->dg_perm, false);
                else launch_small_lu<float>(c, (float *)c->face_pool, 9, 3, 3, c->cells, c->face_perm, false);
            } else {
                if (dg) DGH_DISPATCH_N(c->n, {
                        k1_dg_assemble<N, double><<<grid1(tot), K1_THREADS, 0, c->stream>>>(
                            (double *)c->dg_pool, c->vol, c->fcache, c->b1, c->g1, c->inv_step, 0, c->cells);
                    })
                else k1_face_blocks<double><<<grid1(tot), K1_THREADS, 0, c->stream>>>(c->S, c->speeds, (double *)c->face_pool, c->g1);
                c->launched();
                if (dg) launch_small_lu<double>(c, (double *)c->dg_pool, (size_t)c->m * c->m, c->m, c->m, c->cells, c->dg_perm, false);
                else launch_small_lu<double>(c, (double *)c->face_pool, 9, 3, 3, c->cells, c->face_perm, false);
            }
            c->check_status();
            (dg ? c->dg_factored : c->face_factored) = true;
            return;
        }
        if (op == DGH_OP_DG && c->ilu2d()) {
            need(c->ilu2.on, "context has no DG operator");
            need(c->linearised, "Refresh the volume Jacobian before assembling a block");
            if (c->mixed()) ilu2_factor<float>(c);
            else ilu2_factor<double>(c);
            c->check_status();
            c->dg_factored = true;
        } else if (op == DGH_OP_DG) {
            need(c->dg_pool, "context has no DG operator");
            need(c->linearised, "Refresh the volume Jacobian before assembling a block");
            if (c->dg_variant < 0 && c->half16()) c->dg_variant = 0;  // one factorisation form
            if (c->dg_variant < 0) {
                const int sample = std::min(c->cells, std::max(c->lu_grid, 1) * 4);
                c->dg_variant = tuned_variant_all(c, 0, [&](int v) { dg_factor(c, v, 0, sample); }, c->tune_ms);
                c->check_status();
            }
            if (c->fused_ctas < 0) {  // the fused path's residency (kind 4): 1 or 2 CTAs per SM
                const bool fused = c->mixed() && (c->half16() || c->dg_variant == 0) && !c->overint();
                if (fused) {
                    const int sample = std::min(c->cells, std::max(c->lu_grid, 1) * 4);
                    const int v = tuned_variant_all(c, 4, [&](int k) {
                        c->fused_ctas = k + 1;
                        dg_factor(c, c->dg_variant, 0, sample);
                    }, c->fused_ms);
                    c->fused_ctas = c->cfg.autotune ? v + 1 : 2;
                    c->check_status();
                } else {
                    c->fused_ctas = 2;
                }
            }
            dg_factor(c, c->dg_variant, 0, c->cells);
            c->check_status();
            c->dg_factored = true;
            if (c->solve_shape < 0) {  // timed on a zero right-hand side (the same loads and flops)
                ck(cudaMemsetAsync(c->gw, 0, (size_t)c->N * sizeof(double), c->stream), "cudaMemsetAsync");
                c->solve_shape = tuned_variant_all(c, 3, [&](int v) { dg_block_solve(c, v, c->gw, c->gz); }, c->solve_ms);
            }
        } else {
            need(c->face_pool, "context has no HDG operator");
            need(c->condensed, "Condense the HDG operator before refreshing its preconditioner");
            const long long tot = (long long)c->faces * c->fw * c->fw;
            const size_t stride = (size_t)c->fw * c->fw;
            c->face_inverse = false;
            if (c->mixed() && c->fw <= 64 && (size_t)tot * sizeof(double) <= c->aug_bytes) {
                // FP64 blocks in the condensation workspace (free until the next condensation),
                // inverted in FP64 and stored as FP32 inverses
                face_blocks<double>(c, c->aug);
                const size_t smem = inv_narrow_smem_bytes(c->fw);
                allow_dynamic_smem((const void *)k_inv_narrow, smem);
                int resident = 0;
                ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, k_inv_narrow, INV_THREADS, smem), "occupancy");
                constexpr int wpc = INV_THREADS / 32;
                const int grid = std::min((c->faces + wpc - 1) / wpc, c->sms * std::max(1, resident));
                k_inv_narrow<<<grid, INV_THREADS, smem, c->stream>>>(c->aug, c->fw, c->faces, (float *)c->face_pool,
                                                                     c->status, ST_SINGULAR);
                c->launched();
                c->face_inverse = true;
            } else if (c->mixed()) {
                face_blocks<float>(c, (float *)c->face_pool);
                launch_lu_narrow<float>(c, (float *)c->face_pool, c->fw, c->faces, c->face_perm, ST_SINGULAR);
            } else {
                face_blocks<double>(c, (double *)c->face_pool);
                launch_lu_narrow<double>(c, (double *)c->face_pool, c->fw, c->faces, c->face_perm, ST_SINGULAR);
            }
            c->check_status();
            c->face_factored = true;
        }
    });
}
int dgh_precond_apply(dgh_ctx *c, int op, const double *x, double *z) {
    return guard(c, [&] { precond_apply(c, op, x, z); });
}

// ---- HybridOperator ------------------------------------------------------------------------------
int dgh_hdg_refresh_projected(dgh_ctx *c, const double *u, const double *r) {
    return guard(c, [&] {
        need(c->has_hdg(), "context has no HDG operator");
        Timed tm(c, DGH_TIMER_CONDENSE);
        slab_halo(c, r);  // the ghost cells are condensed too, with their own residual rows
        linearise(c, u);
        const int ld = c->m + c->t + 1;
        if (c->d1()) {
            // dg_hdg_1d/src/hybrid.cpp:39-84: [A | B | r] per cell, LU + back substitution, S and C y
            for (int first = 0; first < c->cells; first += c->aug_cells) {
                const int count = std::min(c->aug_cells, c->cells - first);
                DGH_DISPATCH_N(c->n, {
                    k1_hdg_assemble<N><<<grid1((long long)count * c->m * ld), K1_THREADS, 0, c->stream>>>(
                        c->aug, c->vol, c->traces, c->speeds, r, c->b1, c->g1, c->inv_step, first, count);
                });
                c->launched();
                launch_small_lu<double>(c, c->aug, (size_t)c->m * ld, c->m, ld, count, c->aug_perm, true);
                DGH_DISPATCH_N(c->n, {
                    k1_hdg_schur<N><<<grid1((long long)count * T1 * (T1 + 1)), K1_THREADS, 0, c->stream>>>(
                        c->aug, c->traces, c->speeds, c->S, c->X, c->Y, c->cy, c->b1, c->g1, first, count);
                });
                c->launched();
            }
            k1_hdg_rhs<<<grid1(c->NT), K1_THREADS, 0, c->stream>>>(c->cy, c->hrhs, c->g1);
            c->launched();
            c->check_status();
            c->condensed = true;
            return;
        }
        if (c->c32()) {
            // variant 0: FP64 tensor-pipe LU, FP32 storage; 1: FP32 LU (autotuned per degree)
            auto chunk = [&](int v, int first, int count) {
                if (v == 0) hdg_condense_chunk32_tc(c, r, first, count);
                else hdg_condense_chunk32(c, r, first, count);
            };
            if (c->hdg_variant < 0) {
                const int sample = std::min(aug_chunk<double>(c), std::max(c->lu_grid, 1) * 4);
                c->hdg_variant = tuned_variant_all(c, 2, [&](int v) { chunk(v, 0, sample); }, c->tune_ms + 2);
                c->check_status();
            }
            const int per = c->hdg_variant == 0 ? aug_chunk<double>(c) : aug_chunk<float>(c);
            for (int first = 0; first < c->cells; first += per)
                chunk(c->hdg_variant, first, std::min(per, c->cells - first));
            hdg_rhs_from_cy(c);
            c->check_status();
            c->condensed = true;
            return;
        }
        if (c->hdg_variant < 0) {
            const int sample = std::min(c->aug_cells, std::max(c->lu_grid, 1) * 4);
            c->hdg_variant = tuned_variant_all(c, 1, [&](int v) { hdg_condense_chunk(c, v, r, 0, sample); }, c->tune_ms + 2);
            c->check_status();
        }
        for (int first = 0; first < c->cells; first += c->aug_cells)
            hdg_condense_chunk(c, c->hdg_variant, r, first, std::min(c->aug_cells, c->cells - first));
        DGH_DISPATCH_N(c->n, {
            const long long tot = c->NT;
            k_hdg_rhs<N><<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(c->cy, c->hrhs, c->g);
        });
        c->launched();
        c->check_status();
        c->condensed = true;
    });
}
int dgh_hdg_rhs(dgh_ctx *c, double *rhs) {
    return guard(c, [&] {
        need(c->condensed, "Condense the HDG operator first");
        ck(cudaMemcpyAsync(rhs, c->hrhs, c->NT * sizeof(double), cudaMemcpyDeviceToDevice, c->stream), "copy");
        slab_zero_ghost_faces(c, rhs);
    });
}
int dgh_hdg_apply(dgh_ctx *c, const double *lam, double *out) {
    return guard(c, [&] { hdg_apply(c, lam, out); });
}
int dgh_hdg_block(dgh_ctx *c, int row, int col, double *host_block) {
    return guard(c, [&] {
        need(c->condensed, "Condense the HDG operator first");
        need(row == col && row >= 0 && row < c->faces, "Only diagonal face blocks are exposed on the device");
        const long long tot = (long long)c->faces * c->fw * c->fw;
        double *tmp = c->alloc<double>(tot);
        if (c->d1()) {
            k1_face_blocks<double><<<grid1(tot), K1_THREADS, 0, c->stream>>>(c->S, c->speeds, tmp, c->g1);
            c->launched();
        } else {
            face_blocks<double>(c, tmp);
        }
        ck(cudaMemcpyAsync(host_block, tmp + (size_t)row * c->fw * c->fw, (size_t)c->fw * c->fw * sizeof(double),
                           cudaMemcpyDeviceToHost, c->stream), "copy");
        c->sync();
        ck(cudaFree(tmp), "cudaFree");
        c->owned.pop_back();
        c->bytes -= std::max<size_t>(tot * sizeof(double), 16);
    });
}
int dgh_hdg_recover(dgh_ctx *c, const double *dl, double *du) {
    return guard(c, [&] {
        need(c->condensed, "Condense the HDG operator first");
        slab_trace_halo(c, dl);
        if (c->d1()) {
            DGH_DISPATCH_N(c->n, { k1_hdg_recover<N><<<grid1(c->N), K1_THREADS, 0, c->stream>>>(c->X, c->Y, dl, du, c->g1); });
        } else if (c->c32()) {
            // du = A^{-1} (-B dlambda) - y with the kept FP32 factors (= -X dlambda - y)
            DGH_DISPATCH_N(c->n, {
                const long long tot = (long long)c->cells * N * N;
                k_hdg_bmul<N><<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(dl, c->speeds, c->hq, c->basis, c->g);
            });
            c->launched();
            launch_solve<float>(c, c->lu32, c->lu32_perm, (size_t)c->m * c->m, c->m, c->cells, c->hq, du);
            axpby(c, 1., du, -1., c->Y, du, c->N);
            return;
        } else {
            DGH_DISPATCH_N(c->n, { k_hdg_recover<N><<<c->cells, 256, 0, c->stream>>>(c->X, c->Y, dl, du, c->g); });
        }
        c->launched();
    });
}
int dgh_hdg_retarget(dgh_ctx *c, const double *r) {
    return guard(c, [&] {
        need(c->condensed, "Condense the HDG operator first");
        need(c->c32(), "Retargeting needs the kept FP32 cell factors (condense32)");
        Timed tm(c, DGH_TIMER_CONDENSE);
        slab_halo(c, r);
        // y = A^{-1} r with the kept factors, C y per cell, and the condensed right-hand side
        launch_solve<float>(c, c->lu32, c->lu32_perm, (size_t)c->m * c->m, c->m, c->cells, r, c->Y);
        DGH_DISPATCH_N(c->n, {
            k_hdg_schur<N, double, true, float><<<std::min(c->cells, c->sms * 8), 256, 0, c->stream>>>(
                nullptr, c->fcache, c->speeds, nullptr, nullptr, c->Y, c->cy, c->basis, c->g, 0, c->cells,
                NFACES * NVAR * N);
        });
        c->launched();
        hdg_rhs_from_cy(c);
    });
}
int dgh_hdg_recovered_residual(dgh_ctx *c, const double *e, double *out) {
    return guard(c, [&] {
        need(c->condensed, "Condense the HDG operator first");
        slab_trace_halo(c, e);
        if (c->d1()) {
            DGH_DISPATCH_N(c->n, {
                k1_hdg_recovered_residual<N><<<grid1(c->N), K1_THREADS, 0, c->stream>>>(e, c->speeds, out, c->b1, c->g1);
            });
            c->launched();
            return;
        }
        DGH_DISPATCH_N(c->n, {
            const long long tot = (long long)c->cells * N * N;
            k_hdg_recovered_residual<N><<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(e, c->speeds, out, c->basis, c->g);
        });
        c->launched();
    });
}

// ---- GMRES -------------------------------------------------------------------------------------------
int dgh_gmres(dgh_ctx *c, int op, const double *rhs, double *x, int limit, double tol, int *iterations, double *relative) {
    return guard(c, [&] {
        need(op >= 0 && op <= 2, "Invalid operator");
        need(op == DGH_OP_HDG ? c->has_hdg() : c->has_dg(), "context lacks the requested operator");
        int it = 0;
        double rel = 0;
        try {
            gmres(c, op, rhs, x, limit, tol, it, rel);
        } catch (...) {
            if (iterations) *iterations = it;
            throw;
        }
        if (iterations) *iterations = it;
        if (relative) *relative = rel;
    });
}
int dgh_shape_set(dgh_ctx *c, int which, int value) {
    if (!c) return DGH_ERR_INVALID;
    if (which == DGH_SHAPE_SOLVE_GRID && (value == 0 || value == 1)) c->solve_shape = value;
    else if (which == DGH_SHAPE_FUSED_CTAS && (value == 1 || value == 2)) c->fused_ctas = value;
    else return DGH_ERR_INVALID;
    return DGH_OK;
}
int dgh_autotune_shapes(const dgh_ctx *c, double out[6]) {
    if (!c || !out) return DGH_ERR_INVALID;
    out[0] = c->solve_shape;
    out[1] = c->solve_ms[0];
    out[2] = c->solve_ms[1];
    out[3] = c->fused_ctas;
    out[4] = c->fused_ms[0];
    out[5] = c->fused_ms[1];
    return DGH_OK;
}
int dgh_autotune_report(const dgh_ctx *c, double out[6]) {
    if (!c || !out) return DGH_ERR_INVALID;
    out[0] = c->dg_variant;
    out[1] = c->hdg_variant;
    for (int i = 0; i < 4; ++i) out[2 + i] = c->tune_ms[i];
    return DGH_OK;
}
int dgh_gmres_graph_enable(dgh_ctx *c, int on) {
    return guard(c, [&] {
        need(!on || !c->slabbed(), "Slab contexts launch their GMRES cycles step by step");
        c->use_graph = on != 0;
    });
}
const double *dgh_gmres_residual(dgh_ctx *c, int op) {
    if (!c || op < 0 || op > 2) return nullptr;
    return c->gres[op];
}

}  // extern "C"

// ---- Standalone block Jacobi (BlockJacobi, block_jacobi.hpp:7-47) -----------------------------------
// A pool of `count` dense m x m blocks, factored by one of the device LU kernels and applied as
// z = A^{-1} x per block.  It runs on a bare context that carries only what the launch helpers
// read: the stream, the status word, the SM count and the left-looking kernel's scratch.
struct dgh_block_jacobi {
    dgh_ctx *c = nullptr;
    int m = 0, count = 0, precision = 0, variant = 0;
    void *pool = nullptr;
    int *perm = nullptr;
    double *ws = nullptr;  // FP64 workspace of the left-looking kernel in the mixed form
    bool factored = false;
};

extern "C" {

int dgh_block_jacobi_create(int m, int count, int precision, int variant, int device, dgh_block_jacobi **out) {
    if (!out) return DGH_ERR_INVALID;
    *out = nullptr;
    auto *bj = new dgh_block_jacobi;
    bj->c = new dgh_ctx;
    dgh_ctx *c = bj->c;
    const int rc = guard(c, [&] {
        need(m >= 1 && count >= 1 && m <= 2 * LL_THREADS, "Invalid block size or count");
        need(precision == DGH_PRECISION_FP64 || precision == DGH_PRECISION_MIXED, "Invalid precision");
        need(variant >= 0 && variant <= 3, "Invalid factorisation variant");
        need(variant != 0 || m % 4 == 0, "LU block width unsupported by the left-looking kernel");
        need(variant < 2 || (m <= 64 && m % 4 == 0), "block width unsupported by the narrow LU");
        need(variant != 3 || precision == DGH_PRECISION_MIXED, "explicit inverses are the mixed form only");
        need(m % 4 == 0, "block width must be a multiple of 4 (slab layout)");
        bj->m = m;
        bj->count = count;
        bj->precision = precision;
        bj->variant = variant;
        c->cfg.precision = precision;
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) fail(DGH_ERR_CUDA, "no CUDA device available");
        ck(cudaSetDevice(device), "cudaSetDevice");
        cudaDeviceProp prop{};
        ck(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
        if (prop.major < 10) fail(DGH_ERR_CUDA, "this library is built for sm_100a (B200) only");
        c->sms = prop.multiProcessorCount;
        c->red_grid = c->sms * RED_BLOCKS_PER_SM;
        ck(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        ck(cudaMallocHost((void **)&c->pinned, 4096), "cudaMallocHost");
        c->status = c->alloc<int>(1);
        ck(cudaMemset(c->status, 0, sizeof(int)), "memset");
        const size_t tsz = precision == DGH_PRECISION_MIXED ? sizeof(float) : sizeof(double);
        bj->pool = c->alloc<char>((size_t)count * m * m * tsz);
        bj->perm = c->alloc<int>((size_t)count * m);
        if (variant == 0) {
            const size_t smem = lu_left_smem_bytes(m);
            allow_dynamic_smem((const void *)k_lu_left<false>, smem);
            int per_sm = 0;
            ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lu_left<false>, LL_THREADS, smem), "occupancy");
            c->lu_grid = c->sms * std::max(1, per_sm);
            c->lu_tri = c->alloc<double>((size_t)c->lu_grid * ((m + LL_NB - 1) / LL_NB) * LL_TRI);
        }
        if (precision == DGH_PRECISION_MIXED && (variant == 0 || variant == 3))
            bj->ws = c->alloc<double>((size_t)count * m * m);
        c->sync();
    });
    if (rc != DGH_OK) {
        g_create_error = c->err;
        dgh_block_jacobi_destroy(bj);
        return rc;
    }
    *out = bj;
    return DGH_OK;
}

int dgh_block_jacobi_destroy(dgh_block_jacobi *bj) {
    if (!bj) return DGH_OK;
    dgh_ctx_destroy(bj->c);
    delete bj;
    return DGH_OK;
}

const char *dgh_block_jacobi_error(const dgh_block_jacobi *bj) {
    return bj ? bj->c->err.c_str() : g_create_error.c_str();
}

int dgh_block_jacobi_factor(dgh_block_jacobi *bj, const double *blocks) {
    if (!bj) return DGH_ERR_INVALID;
    dgh_ctx *c = bj->c;
    return guard(c, [&] {
        need(blocks != nullptr, "null block pointer");
        const int m = bj->m, count = bj->count;
        const size_t stride = (size_t)m * m, bytes = stride * count * sizeof(double);
        bj->factored = false;
        if (bj->precision == DGH_PRECISION_FP64) {
            double *pool = (double *)bj->pool;
            ck(cudaMemcpyAsync(pool, blocks, bytes, cudaMemcpyDeviceToDevice, c->stream), "copy blocks");
            if (bj->variant == 0) launch_lu_left<false>(c, pool, stride, m, m, count, bj->perm, ST_SINGULAR, true);
            else if (bj->variant == 1) launch_lu<double>(c, pool, stride, m, m, count, bj->perm, ST_SINGULAR, true);
            else launch_lu_narrow<double>(c, pool, m, count, bj->perm, ST_SINGULAR);
        } else {
            float *pool = (float *)bj->pool;
            if (bj->variant == 0 || bj->variant == 3) {
                ck(cudaMemcpyAsync(bj->ws, blocks, bytes, cudaMemcpyDeviceToDevice, c->stream), "copy blocks");
                if (bj->variant == 0) {
                    launch_lu_left<false>(c, bj->ws, stride, m, m, count, bj->perm, ST_SINGULAR, false, pool);
                } else {
                    const size_t smem = inv_narrow_smem_bytes(m);
                    allow_dynamic_smem((const void *)k_inv_narrow, smem);
                    int resident = 0;
                    ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, k_inv_narrow, INV_THREADS, smem),
                       "occupancy");
                    constexpr int wpc = INV_THREADS / 32;
                    const int grid = std::min((count + wpc - 1) / wpc, c->sms * std::max(1, resident));
                    k_inv_narrow<<<grid, INV_THREADS, smem, c->stream>>>(bj->ws, m, count, pool, c->status, ST_SINGULAR);
                    c->launched();
                }
            } else {
                k_round<<<(unsigned)std::min<long long>(((long long)stride * count + 255) / 256, 65535LL * 16), 256, 0,
                          c->stream>>>(blocks, pool, (long long)stride * count);
                c->launched();
                if (bj->variant == 1) launch_lu<float>(c, pool, stride, m, m, count, bj->perm, ST_SINGULAR, true);
                else launch_lu_narrow<float>(c, pool, m, count, bj->perm, ST_SINGULAR);
            }
        }
        c->check_status();
        bj->factored = true;
    });
}

int dgh_block_jacobi_apply(dgh_block_jacobi *bj, const double *x, double *z) {
    if (!bj) return DGH_ERR_INVALID;
    dgh_ctx *c = bj->c;
    return guard(c, [&] {
        need(bj->factored, "Refresh the block-Jacobi preconditioner before applying it");
        const int m = bj->m, count = bj->count;
        const size_t stride = (size_t)m * m;
        if (bj->variant == 3) {
            constexpr int wpc = INV_APPLY_THREADS / 32;
            const int grid = std::min((count + wpc - 1) / wpc, c->sms * 8);
            k_inv_apply<<<grid, INV_APPLY_THREADS, 0, c->stream>>>((const float *)bj->pool, m, count, x, z);
            c->launched();
        } else if (bj->precision == DGH_PRECISION_MIXED) {
            launch_solve<float>(c, (const float *)bj->pool, bj->perm, stride, m, count, x, z);
        } else {
            launch_solve<double>(c, (const double *)bj->pool, bj->perm, stride, m, count, x, z);
        }
        c->sync();
    });
}

int dgh_block_jacobi_perm(const dgh_block_jacobi *bj, int *host_perm) {
    if (!bj || !host_perm) return DGH_ERR_INVALID;
    dgh_ctx *c = bj->c;
    return guard(c, [&] {
        need(bj->factored && bj->variant != 3, "no factored permutation");
        ck(cudaMemcpy(host_perm, bj->perm, sizeof(int) * (size_t)bj->m * bj->count, cudaMemcpyDeviceToHost),
           "copy perm");
    });
}

}  // extern "C"

// ---- lockstep batch of DG GMRES solves (no counterpart in the reference) ------------------------
namespace {
thread_local std::string g_ls_error;
void ls_free(dgh_lockstep *L) {
    if (L->stream) cudaStreamSynchronize(L->stream);
    for (dgh_ctx *c : L->members) {
        c->ls = nullptr;
        c->ls_index = -1;
    }
    for (auto &sl : L->slots)
        if (sl.ready) cudaEventDestroy(sl.ready);
    if (L->finished) cudaEventDestroy(L->finished);
    if (L->table) cudaFree(L->table);
    if (L->flags) cudaFree(L->flags);
    if (L->tails) cudaFree(L->tails);
    if (L->host) cudaFreeHost(L->host);
    if (L->flags_host) cudaFreeHost(L->flags_host);
    if (L->tails_host) cudaFreeHost(L->tails_host);
    if (L->cycle) cudaGraphExecDestroy(L->cycle);
    if (L->aux) cudaStreamDestroy(L->aux);
    if (L->stream) cudaStreamDestroy(L->stream);
    delete L;
}
}  // namespace

extern "C" {

const char *dgh_lockstep_error(void) { return g_ls_error.c_str(); }

int dgh_lockstep_create(dgh_ctx *const *members, int count, dgh_lockstep **out) {
    return dgh_lockstep_create_op(members, count, DGH_OP_DG, out);
}

int dgh_lockstep_create_op(dgh_ctx *const *members, int count, int op, dgh_lockstep **out) {
    if (!members || count <= 0 || !out || (op != DGH_OP_DG && op != DGH_OP_HDG)) return DGH_ERR_INVALID;
    const bool hdg = op == DGH_OP_HDG;
    *out = nullptr;
    auto reject = [&](int i, const char *m) {
        g_ls_error = "lockstep member " + std::to_string(i) + ": " + m;
        return DGH_ERR_INVALID;
    };
    for (int i = 0; i < count; ++i) {
        const dgh_ctx *c = members[i];
        if (!c) return reject(i, "null context");
        if (c->d1()) return reject(i, "lockstep members are 2D contexts");
        if (!hdg && !c->has_dg()) return reject(i, "the context has no DG operator");
        if (hdg && !c->has_hdg()) return reject(i, "the context has no HDG operator");
        if (c->overint()) return reject(i, "lockstep members use the collocated volume rule");
        if (c->ilu()) return reject(i, "lockstep members use block Jacobi");
        if (c->slabbed()) return reject(i, "slab contexts solve on their own");
        if (c->ls) return reject(i, "the context is already in a lockstep group");
        for (int k = 0; k < i; ++k)
            if (members[k] == c) return reject(i, "the context is listed twice");
        const dgh_ctx *c0 = members[0];
        if (c->cfg.device != c0->cfg.device) return reject(i, "lockstep members share one device");
        if (c->cfg.precision != c0->cfg.precision) return reject(i, "lockstep members share one precision");
        const long long n = hdg ? c->NT : c->N, n0 = hdg ? c0->NT : c0->N;
        if (std::min<long long>(n, c->cfg.restart) != std::min<long long>(n0, c0->cfg.restart))
            return reject(i, "lockstep members share one GMRES restart length");
    }
    auto *L = new dgh_lockstep;
    const int rc = [&]() -> int {
        try {
            const dgh_ctx *c0 = members[0];
            L->device = c0->cfg.device;
            L->precision = c0->cfg.precision;
            L->op = op;
            L->restart = (int)std::min<long long>(hdg ? c0->NT : c0->N, c0->cfg.restart);
            ck(cudaSetDevice(L->device), "cudaSetDevice");
            std::vector<int> order(count);
            for (int i = 0; i < count; ++i) order[i] = i;
            std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return members[a]->n < members[b]->n; });
            for (int i : order) L->members.push_back(members[i]);
            ck(cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking), "cudaStreamCreate");
            ck(cudaEventCreateWithFlags(&L->finished, cudaEventDisableTiming), "cudaEventCreate");
            L->slots.resize(count);
            for (auto &sl : L->slots) ck(cudaEventCreateWithFlags(&sl.ready, cudaEventDisableTiming), "cudaEventCreate");
            ck(cudaMalloc(&L->table, sizeof(LsMember) * count), "cudaMalloc");
            ck(cudaMalloc(&L->flags, sizeof(int) * count), "cudaMalloc");
            ck(cudaMalloc(&L->tails, sizeof(LsTail) * count), "cudaMalloc");
            ck(cudaMallocHost(&L->host, sizeof(LsMember) * count), "cudaMallocHost");
            ck(cudaMallocHost(&L->flags_host, sizeof(int) * count), "cudaMallocHost");
            ck(cudaMallocHost(&L->tails_host, sizeof(LsTail) * count), "cudaMallocHost");
            constexpr int wpc = SOLVE_THREADS / 32;
            auto layout_of = [&](const dgh_ctx *c) { return c->half16() ? 3 : !c->mixed() ? 0 : c->m < 64 ? 2 : 1; };
            for (int i = 0; i < count; ++i) {
                dgh_ctx *c = L->members[i];
                LsMember &t = L->host[i];
                std::memset(&t, 0, sizeof(t));
                t.gdev = c->gdev;
                t.V = c->V;
                t.w = c->gw;
                t.z = c->gz;
                t.red = c->red;
                t.partial = c->partial;
                t.coef = c->gcoef;
                t.x = c->g_x;
                t.rhs = c->g_rhs;
                t.r = c->gres[op];
                t.W = hdg ? c->inv_trace_mass : c->inv_mass;
                t.ld = (size_t)c->vld;
                t.n = hdg ? c->NT : c->N;
                t.red_blocks = c->red_grid;
                t.red0 = L->red_total;
                L->red_total += c->red_grid;
                t.pool = c->dg_pool;
                t.scale = c->dg_scale;
                t.perm = c->dg_perm;
                t.stride = (size_t)c->m * c->m;
                t.m = c->m;
                t.cells = c->cells;
                t.traces = c->traces2;
                t.vol = c->vol;
                t.fcache = c->fcache;
                t.speeds = c->speeds;
                t.basis = c->basis_dev;
                t.g = c->g;
                t.inv_step = c->inv_step;
                // ranges: one per degree (J·v) and one per factor layout (block solve)
                if (L->degrees.empty() || L->degrees.back().key != c->n) {
                    dgh_lockstep::Range r;
                    r.first = i;
                    r.key = c->n;
                    L->degrees.push_back(r);
                }
                auto &dr = L->degrees.back();
                t.team0 = dr.blocks;
                ++dr.count;
                if (hdg) {  // the Schur apply: a CTA per face; the face preconditioner is planned per session
                    dr.blocks += c->faces;
                    t.S = c->c32() ? (const void *)c->S32 : (const void *)c->S;
                    t.c32 = c->c32() ? 1 : 0;
                    t.stride = (size_t)c->fw * c->fw;
                    t.m = c->fw;
                    t.cells = c->faces;
                    continue;
                }
                int cpb = 1;
                DGH_DISPATCH_N(c->n, { cpb = Team<N>::CPB; });
                dr.blocks += c->team_blocks(cpb);
                const int key = layout_of(c);
                if (L->layouts.empty() || L->layouts.back().key != key) {
                    dgh_lockstep::Range r;
                    r.first = i;
                    r.key = key;
                    L->layouts.push_back(r);
                }
                auto &lr = L->layouts.back();
                t.solve0 = lr.blocks;
                lr.blocks += (c->cells + wpc - 1) / wpc;
                ++lr.count;
                const size_t row = key == 3 ? sizeof(float) * pad8(c->m) : (key == 0 ? sizeof(double) : sizeof(float)) * c->m;
                lr.smem = std::max(lr.smem, row * wpc);
            }
            for (const auto &r : L->layouts)
                for (const auto &q : L->layouts)
                    if (&r != &q && r.key == q.key) fail(DGH_ERR_INVALID, "lockstep factor layouts are not contiguous");
            for (int i = 0; i < count; ++i) {
                L->members[i]->ls = L;
                L->members[i]->ls_index = i;
            }
            return DGH_OK;
        } catch (const Failure &e) {
            g_ls_error = e.message;
            return e.code;
        } catch (const std::exception &e) {
            g_ls_error = e.what();
            return DGH_ERR_CUDA;
        }
    }();
    if (rc != DGH_OK) {
        for (dgh_ctx *c : L->members) c->ls = nullptr;
        L->members.clear();
        ls_free(L);
        return rc;
    }
    *out = L;
    return DGH_OK;
}

int dgh_lockstep_destroy(dgh_lockstep *L) {
    if (!L) return DGH_ERR_INVALID;
    ls_free(L);
    return DGH_OK;
}

int dgh_lockstep_begin(dgh_lockstep *L, int expected) {
    if (!L || expected < 0 || expected > (int)L->members.size()) return DGH_ERR_INVALID;
    std::lock_guard<std::mutex> lk(L->mu);
    if (L->open) return DGH_ERR_STATE;
    for (auto &sl : L->slots) {
        sl.arrived = sl.withdrawn = sl.trivial = false;
        sl.code = DGH_OK;
        sl.msg.clear();
    }
    L->arrived = L->withdrawn = 0;
    L->expected = expected;
    L->open = expected > 0;
    return DGH_OK;
}

int dgh_lockstep_leave(dgh_lockstep *L, dgh_ctx *c) {
    if (!L || !c || c->ls != L) return DGH_ERR_INVALID;
    std::unique_lock<std::mutex> lk(L->mu);
    auto &sl = L->slots[c->ls_index];
    if (!L->open || sl.arrived || sl.withdrawn) return DGH_OK;
    sl.withdrawn = true;
    ++L->withdrawn;
    if (L->arrived + L->withdrawn == L->expected) {
        lk.unlock();
        ls_complete(L);
    }
    return DGH_OK;
}

int dgh_lockstep_report(const dgh_lockstep *L, int64_t out[4]) {
    if (!L || !out) return DGH_ERR_INVALID;
    out[0] = L->sessions;
    out[1] = L->cycles;
    out[2] = L->steps;
    out[3] = L->launches;
    return DGH_OK;
}

}  // extern "C"
