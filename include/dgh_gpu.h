/* dgh_gpu.h — C ABI of the B200 (sm_100a) implicit 2D DG / condensed-HDG Euler solver.
 *
 * Drop-in boundary for the reference YueWu2002/DG_HDG_Euler_Cpp.  The reference has no FFI;
 * its internal seams are C++ classes, and each entry point below replaces one of them:
 *   Problem        dg_hdg_2d/include/euler/discretization.hpp:7-45
 *   DGOperator     dg_hdg_2d/include/euler/dg_operator.hpp:5-17
 *   BlockJacobi    common/include/euler/linalg/block_jacobi.hpp:7-47
 *   HybridOperator dg_hdg_2d/include/euler/hybrid.hpp:6-32
 *   GMRES          common/include/euler/linalg/gmres.hpp:21-35
 *   TimeIntegrator dg_hdg_2d/include/euler/time_integrator.hpp:21-40
 *   Config         dg_hdg_2d/include/euler/config.hpp:7-18
 *
 * Conventions
 *  - Every vector argument named u, r, v, x, z, lambda ... is a DEVICE pointer to FP64 data in
 *    the reference layout (types.hpp:22-31 for volume vectors: per cell, NVAR sheets of n*n
 *    nodes with x fastest; discretization.cpp:65-68 for trace vectors: per face NVAR lines of
 *    n values).  Arguments named host_* are host pointers.
 *  - All work is ordered on the context's CUDA stream (dgh_stream).  Functions that return a
 *    host scalar synchronise that stream.
 *  - Every function returns a dgh_status; on failure dgh_last_error() gives the reference's
 *    require() message (e.g. "Singular block Jacobi factor", "GMRES iteration limit reached").
 *  - A context owns all device memory it needs; nothing allocates after dgh_ctx_create except
 *    the optional helpers dgh_vec_alloc/dgh_vec_free.  A context is not thread-safe, as the
 *    reference's operators are not (DESIGN.md:42-43 of the reference).
 *  - There is no CPU fallback: without a usable sm_100 device, dgh_ctx_create fails.
 */
#ifndef DGH_GPU_H
#define DGH_GPU_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dgh_ctx dgh_ctx;

typedef enum dgh_status {
    DGH_OK = 0,
    DGH_ERR_INVALID = 1,      /* bad argument or configuration (config.cpp:6-22)          */
    DGH_ERR_CUDA = 2,         /* CUDA runtime error, no device, or out of device memory    */
    DGH_ERR_SINGULAR = 3,     /* singular or non-finite block factor (block_jacobi.hpp:16) */
    DGH_ERR_NONFINITE = 4,    /* non-finite GMRES residual (gmres.cpp:117)                 */
    DGH_ERR_GMRES_LIMIT = 5,  /* GMRES iteration limit reached (gmres.cpp:121)             */
    DGH_ERR_BREAKDOWN = 6,    /* GMRES Arnoldi breakdown (gmres.cpp:92)                    */
    DGH_ERR_STATE = 7,        /* invalid physical state (physics.cpp:108, discretization)  */
    DGH_ERR_SOLVER = 8,       /* Newton / line search / HDG acceptance failure             */
    DGH_ERR_COMM = 9          /* slab collective failed: a peer rank failed or timed out   */
} dgh_status;

enum { DGH_METHOD_DG = 0, DGH_METHOD_HDG = 1, DGH_METHOD_BOTH = 2 };
enum { DGH_INTEGRATOR_DIRK3 = 0, DGH_INTEGRATOR_BE = 1 };
enum { DGH_TEST_DIAGONAL = 0, DGH_TEST_WAVE = 1, DGH_TEST_AXIS = 2 };
/* Precision of the block-Jacobi factors and their solves.  Residuals, J*v, Arnoldi and the
 * least-squares problem are always FP64 (the Schur apply and the condensation too, unless
 * dgh_config.condense32).  MIXED: FP32 factors and solves.  MIXED16 (2D; no counterpart in the
 * reference, and below the FP32 its mixed-precision plan names): the DG cell factors are computed
 * in FP64 and stored in FP16, each row of U divided by its largest entry (the row scale kept in
 * FP32), and solved in FP32; the HDG face blocks are as in MIXED.  The transposed solve
 * (DGH_OP_DG_T) needs FP64 or FP32 factors. */
enum { DGH_PRECISION_FP64 = 0, DGH_PRECISION_MIXED = 1, DGH_PRECISION_MIXED16 = 2 };
/* Operators for the preconditioner and GMRES: the DG Jacobian J, the condensed Schur operator,
 * and the DG adjoint J^T (with the transposed block-Jacobi preconditioner). */
enum { DGH_OP_DG = 0, DGH_OP_HDG = 1, DGH_OP_DG_T = 2 };

/* config.hpp:7-18 plus the precision and the operators to allocate.  dim = 1 selects the 1D
 * solver of dg_hdg_1d/ (config.hpp:7-19 there): nx is the number of cells, ny is ignored,
 * NVAR = 3, two faces per cell, and quadrature may exceed degree+1 (over-integration, up to
 * 20 points).  In 2D the quadrature is 0 or degree+1 (collocated) or any value from degree+2
 * to 16 (the over-integrated volume rule). */
typedef struct dgh_config {
    int nx, ny, degree, quadrature;
    int restart, max_linear, max_newton, steps, newton_steps, warmup_updates;
    double cfl, final_time, safety, nonlinear_tolerance, linear_tolerance;
    int method;       /* DGH_METHOD_*: which operators the context allocates               */
    int integrator;   /* DGH_INTEGRATOR_*                                                  */
    int testcase;     /* DGH_TEST_*                                                        */
    int precision;    /* DGH_PRECISION_*                                                   */
    int check_update; /* HDG: independent DG J*v check of every update (time_integrator.cpp:153-162) */
    int device;       /* CUDA device ordinal                                               */
    int dim;          /* 2 (dg_hdg_2d, the default) or 1 (dg_hdg_1d)                       */
    int autotune;     /* 2D: time the factorisation variants on the first refresh (per degree) */
    int preconditioner; /* 0 block Jacobi; 1 block ILU(0), natural ordering                   */
                        /* (common/src/linalg/block_ilu.cpp:15-84): 1D, and 2D for method DG  */
                        /* (level-scheduled sweeps; not for the adjoint operator)             */
    int condense32;     /* 2D HDG: 1 = FP32 condensation (see dgh_hdg_retarget); 0 = FP64     */
    int forcing;        /* linear solve stop: 0 = the reference's relative ltol; 1 = also stop */
                        /* at an absolute floor: min(allowance / 2, ntol max(1, r0) sqrt(lx ly) / 10) */
                        /* (time_integrator.cpp:143-147's allowance; no counterpart otherwise) */
} dgh_config;

/* config.hpp:7-18 defaults: nx=ny=8, k=3, restart 30, max_linear 1500, max_newton 30,
 * cfl 2, T 0.2, safety 1.1, ntol = ltol = 1e-12, ssp-dirk3, diagonal test case, both methods,
 * dim 2.  (The 1D program's defaults differ only in cells = 32.) */
void dgh_config_default(dgh_config *cfg);

/* ---- context ----------------------------------------------------------------------------- */
int dgh_ctx_create(const dgh_config *cfg, dgh_ctx **out);
int dgh_ctx_destroy(dgh_ctx *ctx);
const char *dgh_last_error(const dgh_ctx *ctx);
/* sizes[0..7]: volume size, trace size, cell block width m, cells, faces, nodes per direction
 * n, local trace size t, face width fw */
int dgh_sizes(const dgh_ctx *ctx, int64_t sizes[8]);
/* The configuration the context was created with. */
int dgh_get_config(const dgh_ctx *ctx, dgh_config *out);
void *dgh_stream(const dgh_ctx *ctx);       /* the cudaStream_t all work is ordered on */
/* out[0..3] = hx, hy, lx, ly (discretization.cpp:4-8, example.hpp:9-14); in 1D h, 1, 2, 1 so
 * that the physical rms norm / sqrt(lx ly) is dg_hdg_1d's norm / sqrt(2). */
int dgh_geometry(const dgh_ctx *ctx, double out[4]);
/* Gauss nodes and weights on [-1,1] (n values each; either pointer may be NULL) */
int dgh_nodes(const dgh_ctx *ctx, double *x, double *w);
int dgh_sync(dgh_ctx *ctx);
/* Device bytes held by the context (the pools sized at creation). */
int dgh_device_bytes(const dgh_ctx *ctx, int64_t *bytes);
/* Number of kernels this context has launched since creation (for launch accounting). */
int64_t dgh_launch_count(const dgh_ctx *ctx);
/* Optional CUDA-event timers around each class of kernel work (no counterpart in the reference,
 * which times whole Newton updates only: time_integrator.cpp:93,180).  Enabling resets them. */
enum {
    DGH_TIMER_PRECOND = 0,     /* block-Jacobi solves (the per-iteration factor stream)      */
    DGH_TIMER_OPERATOR = 1,    /* J*v or the Schur apply                                    */
    DGH_TIMER_ARNOLDI = 2,     /* CGS2 dots/updates and the basis normalisation             */
    DGH_TIMER_FACTOR = 3,      /* DG block assembly + batched LU                            */
    DGH_TIMER_FACE_FACTOR = 4, /* HDG face-block assembly + batched LU                      */
    DGH_TIMER_CONDENSE = 5,    /* HDG condensation: assembly, LU, back substitution, S, Cy  */
    DGH_TIMER_RESIDUAL = 6,    /* R(u)                                                      */
    DGH_TIMER_COUNT = 7
};
int dgh_timing_enable(dgh_ctx *ctx, int on);
int dgh_timing_read(dgh_ctx *ctx, int category, double *total_ms, int64_t *count);

/* ---- vector helpers (device memory, stream-ordered) ---------------------------------------- */
int dgh_vec_alloc(dgh_ctx *ctx, int64_t n, double **dev);
int dgh_vec_free(dgh_ctx *ctx, double *dev);
int dgh_upload(dgh_ctx *ctx, double *dev, const double *host, int64_t n);
int dgh_download(dgh_ctx *ctx, double *host, const double *dev, int64_t n);
/* out = a*x + b*y (any of x, y, out may alias) */
int dgh_axpby(dgh_ctx *ctx, double a, const double *x, double b, const double *y, double *out, int64_t n);

/* ---- Problem (discretization.hpp:7-45) ------------------------------------------------------ */
int dgh_initial(dgh_ctx *ctx, double *u);                          /* initial_and_error.cpp:4-54 */
int dgh_freeze(dgh_ctx *ctx, const double *u, double *rate);       /* discretization.cpp:163-195; old = u */
int dgh_set_stage(dgh_ctx *ctx, const double *old, double step_size); /* Problem::old, step_size */
int dgh_residual(dgh_ctx *ctx, const double *u, double *r);        /* discretization.cpp:123-140 */
int dgh_admissible(dgh_ctx *ctx, const double *u, int *ok);        /* discretization.cpp:219-233 */
int dgh_trace(dgh_ctx *ctx, const double *u, double *lambda);      /* discretization.cpp:196-210 */
int dgh_dual_norm(dgh_ctx *ctx, const double *r, double *out);     /* sqrt(r^T M^-1 r), time_integrator.cpp:42 */
int dgh_state_norm(dgh_ctx *ctx, const double *u, double *out);    /* sqrt(u^T M u), time_integrator.cpp:45 */
/* Conservation integrals and L2 errors per variable; in 1D (rho, momentum, energy, 0). */
int dgh_integral(dgh_ctx *ctx, const double *u, double out[4]);    /* discretization.cpp:237-243 */
int dgh_l2_error(dgh_ctx *ctx, const double *u, double time, double out[4]); /* initial_and_error.cpp:55-73 */
int dgh_speeds(dgh_ctx *ctx, double *host_ab);                     /* frozen (a,b) per face node (per face in 1D) */
/* Device copies of the frozen speeds, and replaying recorded ones (they replace Problem::freeze's
 * speeds without touching old/step; used to hold the speeds fixed in the discrete adjoint). */
int dgh_copy_speeds(dgh_ctx *ctx, double *dev_ab);
int dgh_set_speeds(dgh_ctx *ctx, const double *dev_ab);
/* out = a M x + b y with the diagonal mass matrix (discretization.cpp:9-13). */
int dgh_mass_axpby(dgh_ctx *ctx, double a, const double *x, double b, const double *y, double *out);
/* value = sum over nodes of M rho^2 (the adjoint objective); grad (may be NULL) = 2 M rho. */
int dgh_rho2(dgh_ctx *ctx, const double *u, double *value, double *grad);  /* 2D only */

/* ---- DGOperator (dg_operator.hpp:5-17) ------------------------------------------------------ */
int dgh_dg_refresh(dgh_ctx *ctx, const double *u);                 /* dg_operator.cpp:6-9 */
int dgh_dg_apply(dgh_ctx *ctx, const double *v, double *jv);       /* dg_operator.cpp:10-21 */
/* Adjoint J^T w of the DG residual's Jacobian at the same linearisation (no counterpart in the
 * reference: the transpose of dg_operator.cpp:10-21 and volume_jacobian.cpp:59-71). */
int dgh_dg_apply_T(dgh_ctx *ctx, const double *w, double *jtw);    /* 2D only */
/* Diagonal block (row == col), copied to the host row-major m x m (dg_operator.cpp:22-48). */
int dgh_dg_block(dgh_ctx *ctx, int row, int col, double *host_block);

/* ---- BlockJacobi / BlockPreconditioner (block_jacobi.hpp:7-47) ---------------------------------------------------- */
/* op DGH_OP_DG: assemble and factor the E cell blocks from the current DG linearisation;
 * op DGH_OP_HDG: the 2E face blocks of the current condensed operator.  dgh_precond_apply with
 * DGH_OP_DG_T applies the transposed cell-block solves (A^{-T}) from the DG factors. */
int dgh_block_jacobi_refresh(dgh_ctx *ctx, int op);
int dgh_precond_apply(dgh_ctx *ctx, int op, const double *x, double *z);

/* ---- HybridOperator (hybrid.hpp:6-32) ------------------------------------------------------- */
int dgh_hdg_refresh_projected(dgh_ctx *ctx, const double *u, const double *r); /* hybrid.cpp:28-30,56-72 */
int dgh_hdg_rhs(dgh_ctx *ctx, double *rhs);                        /* condensed right-hand side */
int dgh_hdg_apply(dgh_ctx *ctx, const double *lambda, double *out); /* hybrid.cpp:73-82 */
int dgh_hdg_block(dgh_ctx *ctx, int row, int col, double *host_block); /* hybrid.cpp:83-96, row == col */
int dgh_hdg_recover(dgh_ctx *ctx, const double *dlambda, double *du); /* hybrid.cpp:97-105 */
int dgh_hdg_recovered_residual(dgh_ctx *ctx, const double *e, double *out); /* hybrid.cpp:106-121 */
/* FP32 condensation (dgh_config.condense32 = 1; no counterpart in the reference, whose
 * condensation is FP64: hybrid.cpp:56-72).  dgh_hdg_refresh_projected then factors every cell
 * matrix A_K in FP32 with FP32 accumulation, keeps those factors, and stores the Schur blocks
 * S_K = -C A_K^{-1} B in FP32 (no X is stored); the Schur apply reads the FP32 blocks with FP64
 * products, and dgh_hdg_recover computes A_K^{-1}(-B dlambda) - y with the kept factors.  The
 * condensed system then approximates the DG linearisation to FP32 accuracy, so the integrator
 * solves the DG Newton system by iterative refinement: after each Schur solve and recovery it
 * forms the true DG residual e = J du + r with the FP64 J*v, and retargets the condensed system
 * to e for the next correction, until the reference's acceptance target holds.
 * dgh_hdg_retarget: y = A_K^{-1} r per cell with the kept factors, C y, and the condensed
 * right-hand side for volume residual r (dgh_hdg_rhs returns it); the factors and S are reused. */
int dgh_hdg_retarget(dgh_ctx *ctx, const double *r);

/* ---- GMRES (gmres.cpp:17-86) ---------------------------------------------------------------- */
/* Right-preconditioned restarted GMRES(restart) with CGS2 in the M^-1 (DG) or inverse trace
 * mass (HDG) inner product, on op with its block-Jacobi preconditioner.  x is overwritten. */
int dgh_gmres(dgh_ctx *ctx, int op, const double *rhs, double *x, int limit, double tol,
              int *iterations, double *relative);
/* Device pointer to the true residual rhs - A x of the last dgh_gmres call on op. */
/* Per-degree autotuner (no counterpart in the reference).  With dgh_config.autotune set, the
 * first DG block-Jacobi refresh and the first HDG condensation of a context time their
 * factorisation variants on a sample of the context's own cells and keep the faster one; the
 * choice is cached per (degree, precision) for the process.  Variants: DG blocks 0 = left-looking
 * FP64 LU on the tensor pipe (FP32 slabs in the mixed form), 1 = right-looking LU (FP32 in the
 * mixed form); condensation 0 = left-looking LU with the fused right-hand-side solve,
 * 1 = right-looking LU then the tensor-pipe back substitution.  All variants compute the same
 * factors up to rounding.  out[0..1] = the DG and condensation variants in use, -1 where the
 * context has not factored yet; out[2..5] = the last tuning times in ms (DG 0, DG 1, HDG 0,
 * HDG 1; 0 where not timed). */
int dgh_autotune_report(const dgh_ctx *ctx, double out[6]);
/* Launch shapes inside a variant, tuned per degree with autotune set (no counterpart in the
 * reference).  DGH_SHAPE_SOLVE_GRID: the grid of the 2D DG block-Jacobi solves, 0 = every
 * resident CTA slot, 1 = the fewest CTAs with the same number of rounds of blocks per warp (equal
 * shares); timed at the first DG refresh on the context's own factors, cached per (degree,
 * precision, cell count); default 0.  DGH_SHAPE_FUSED_CTAS: CTAs per SM of the fused reduced-
 * precision DG factorisation, 1 (each CTA's FP64 slot fits L2) or 2 (twice the warps); timed at
 * the first DG refresh on a sample of the cells, cached per (degree, precision); default 2.
 * dgh_shape_set fixes a shape instead; every shape computes the same bits.
 * dgh_autotune_shapes: out[0] = the solve grid shape in use (-1 before the first DG refresh),
 * out[1..2] its tuning times (ms) for shapes 0 and 1; out[3] = the fused CTAs per SM in use
 * (-1 before), out[4..5] its tuning times for 1 and 2 (0 where not timed). */
enum { DGH_SHAPE_SOLVE_GRID = 0, DGH_SHAPE_FUSED_CTAS = 1 };
int dgh_autotune_shapes(const dgh_ctx *ctx, double out[6]);
int dgh_shape_set(dgh_ctx *ctx, int which, int value);
/* Replay each GMRES restart cycle as one CUDA graph (its Arnoldi steps are conditional nodes
 * that stop at the reference's inner-loop break, gmres.cpp:65-67) instead of launching it step
 * by step with a host read of the continue flag after every step.  Both ways run the same
 * kernels and give the same results; the graph removes the per-step host round trip.  Off by
 * default.  No counterpart in the reference. */
int dgh_gmres_graph_enable(dgh_ctx *ctx, int on);
const double *dgh_gmres_residual(dgh_ctx *ctx, int op);

/* ---- TimeIntegrator (time_integrator.hpp:21-40, time_integrator.cpp:48-213) ------------------ */
typedef struct dgh_update_stats { /* time_integrator.hpp:9-13 */
    int step, stage, iteration, krylov_iterations;
    double time, stage_time, dt, cfl, residual_physical_rms, damping;
    double linear_relative_residual, dg_linear_relative_residual, iteration_s;
} dgh_update_stats;
typedef struct dgh_run_stats { /* time_integrator.hpp:14-20 */
    double final_time, conservation_drift, seconds, max_linear_residual;
    double max_dg_linear_residual, minimum_step, maximum_step, measured_newton_seconds;
    int steps, newton_iterations, krylov_iterations, measured_updates, updates_recorded;
} dgh_run_stats;

typedef struct dgh_integrator dgh_integrator;
int dgh_integrator_create(dgh_ctx *ctx, int method, dgh_integrator **out);
int dgh_integrator_destroy(dgh_integrator *it);
/* Message of the integrator's last failure (the reference's require() text). */
const char *dgh_integrator_error(const dgh_integrator *it);
/* Full run (TimeIntegrator::advance); host_solution is read and overwritten on the host.
 * Up to max_updates per-update rows are written to updates (may be NULL). */
int dgh_advance(dgh_integrator *it, double *host_solution, dgh_run_stats *stats,
                dgh_update_stats *updates, int max_updates);
/* Speed protocol pieces (speed_test/2d/benchmark.py:21-44): start one backward-Euler stage
 * from a device state (freeze, dt = cfl/rate, old = state), then run single Newton updates
 * (time_integrator.cpp:133-234 for one `it`). */
int dgh_stage_begin(dgh_integrator *it, const double *u, double *dt);
int dgh_newton_update(dgh_integrator *it, dgh_update_stats *stats);
/* The same Newton update through host buffers: host_state is copied to the device first and
 * the updated state is copied back (the end-to-end form of the call). */
int dgh_newton_update_host(dgh_integrator *it, double *host_state, dgh_update_stats *stats);
/* Device pointer to the integrator's current Newton state (size dgh_sizes()[0]). */
double *dgh_integrator_state(dgh_integrator *it);
/* Overrides the reference's fixed limits: the HDG Schur-tolerance attempts (4,
 * time_integrator.cpp:130-149) and the Armijo halvings (30, time_integrator.cpp:165-176).  Lower
 * limits make the failure paths ("Recovered DG residual criterion failed after Schur
 * refinement", "Newton line search failed") reachable from ordinary inputs, for tests. */
int dgh_integrator_set_limits(dgh_integrator *it, int hdg_attempts, int line_search);

/* ---- Standalone block Jacobi (BlockJacobi, common/include/euler/linalg/block_jacobi.hpp:7-47) ----
 * `count` dense m x m blocks (m a multiple of 4, at most 512) factored with row partial pivoting
 * (the first largest |a| wins ties, as LAPACK getrf / Eigen PartialPivLU) by one device LU kernel,
 * then applied as z = A^{-1} x block by block (block_jacobi.hpp:24-39).  blocks, x and z are device
 * pointers; blocks are row-major FP64 and are copied (the caller keeps them).  variant: 0 the
 * left-looking FP64 LU on the tensor pipe, 1 the right-looking blocked LU, 2 the one-warp LU for
 * narrow blocks (m <= 64), 3 FP64 LU with explicit inverses stored in FP32 (m <= 64, mixed only).
 * precision DGH_PRECISION_MIXED stores the factors in FP32 (variant 1 and 2 factor in FP32).  A
 * block with a zero, subnormal or non-finite pivot fails with DGH_ERR_SINGULAR ("Singular block
 * Jacobi factor", block_jacobi.hpp:16-18).  dgh_block_jacobi_perm copies the row permutation
 * (position i of block b holds original row perm[b m + i]). */
typedef struct dgh_block_jacobi dgh_block_jacobi;
int dgh_block_jacobi_create(int m, int count, int precision, int variant, int device, dgh_block_jacobi **out);
int dgh_block_jacobi_destroy(dgh_block_jacobi *bj);
const char *dgh_block_jacobi_error(const dgh_block_jacobi *bj);
int dgh_block_jacobi_factor(dgh_block_jacobi *bj, const double *blocks);
int dgh_block_jacobi_apply(dgh_block_jacobi *bj, const double *x, double *z);
int dgh_block_jacobi_perm(const dgh_block_jacobi *bj, int *host_perm);

/* ---- Batched uneven problems (no counterpart in the reference) ---------------------------------
 * Independent member problems, each with its own dgh_config (mesh, degree, method DG or HDG,
 * precision, restart ...), advanced together on one device.  Every member owns a context and an
 * integrator and is driven by its own host thread, so the members' kernels overlap on the device
 * (each context has its own stream); every member computes exactly what its single-problem run
 * computes.  Calls on a batch are not thread-safe; per-member statuses go to status[] (may be
 * NULL) and the return value is the first failing member's status.
 *   dgh_batch_stage_begin: member i starts a backward-Euler stage from host_states[i] (its
 *     dgh_initial state when host_states or host_states[i] is NULL); dt[i] receives its step.
 *   dgh_batch_newton_update: one Newton update of every member; stats[i] its row. */
typedef struct dgh_batch dgh_batch;
int dgh_batch_create(const dgh_config *members, int count, dgh_batch **out);
int dgh_batch_destroy(dgh_batch *batch);
/* Message of member i's last failure; with batch == NULL the last dgh_batch_create failure. */
const char *dgh_batch_error(const dgh_batch *batch, int member);
int dgh_batch_member(dgh_batch *batch, int member, dgh_ctx **ctx, dgh_integrator **it);
int dgh_batch_stage_begin(dgh_batch *batch, const double *const *host_states, double *dt, int *status);
int dgh_batch_newton_update(dgh_batch *batch, dgh_update_stats *stats, int *status);
/* Member i's current Newton state, copied to the host (size dgh_sizes()[0] of its context). */
int dgh_batch_download(dgh_batch *batch, int member, double *host_state);
/* on = 1: from the next dgh_batch_newton_update on, the 2D members' GMRES solves run in lockstep
 * (dgh_lockstep groups, below: one per class of members sharing method, precision, restart
 * length and device, on the collocated rule with block Jacobi): every phase of an Arnoldi step is
 * one kernel launch over all members of a group; each member's rows stay bitwise those of its
 * own run.  Other members (1D, over-integrated, ILU) keep solving independently.  on = 0
 * returns to independent solves. */
int dgh_batch_lockstep(dgh_batch *batch, int on);
/* The sum of the batch's lockstep groups' dgh_lockstep_report (zeros without any). */
int dgh_batch_lockstep_report(const dgh_batch *batch, int64_t out[4]);

/* ---- Lockstep group of DG GMRES solves (no counterpart in the reference) ------------------------
 * The restart cycles of the DG GMRES solves of several 2D contexts — any degree and mesh size —
 * advanced together: per Arnoldi step one launch of each phase over all members (the block
 * solve once per factor layout present, J*v once per degree present, the CGS2 sweeps,
 * reductions and Givens updates once), each member on its own buffers with its own block
 * partition, so every member's result is bitwise its dgh_gmres result.  Members share device,
 * precision and restart length, use the collocated rule and block Jacobi, and belong to one
 * group at a time; destroy the group before its member contexts.
 * A session: dgh_lockstep_begin(group, expected) opens it for `expected` members; each of them
 * then either calls dgh_gmres(ctx, DGH_OP_DG, ...) (directly or through its integrator) — the
 * call waits until all expected members have arrived, and the last one to arrive issues the
 * lockstep solve on the group's stream — or calls dgh_lockstep_leave(group, ctx) to drop out
 * (a member whose update failed before its solve).  The members' calls come from different host
 * threads (one per member); contexts outside an open session solve independently.
 * dgh_lockstep_report: sessions, restart cycles, Arnoldi steps and kernel launches so far. */
typedef struct dgh_lockstep dgh_lockstep;
int dgh_lockstep_create(dgh_ctx *const *members, int count, dgh_lockstep **out);
/* The same for the solves of operator op: DGH_OP_DG (as above) or DGH_OP_HDG (the condensed
 * Schur solves of 2D contexts with the HDG operator: the Schur apply once per degree, the face
 * preconditioner once per form present, FP32 inverses or LU factors).  An HDG member's first
 * Schur solve of an update joins the session; further solves of the same update (the reference's
 * tolerance retries, FP32-condensation refinement passes) run on their own. */
int dgh_lockstep_create_op(dgh_ctx *const *members, int count, int op, dgh_lockstep **out);
int dgh_lockstep_destroy(dgh_lockstep *group);
const char *dgh_lockstep_error(void);
int dgh_lockstep_begin(dgh_lockstep *group, int expected);
int dgh_lockstep_leave(dgh_lockstep *group, dgh_ctx *member);
int dgh_lockstep_report(const dgh_lockstep *group, int64_t out[4]);

/* ---- Slab domain decomposition (multi-GPU; the reference runs one process on one mesh) ---------
 * One 2D DG or HDG problem split into slabs of whole cell rows, one rank per slab: rank r of `size`
 * owns global rows [row0, row0 + rows) (dgh_slab_rows: ny = size * base + extra, the first
 * `extra` ranks take base + 1 rows; out = {row0, rows, rank below, rank above}, periodic).
 * A slab context (dgh_ctx_create_slab; cfg as for the whole mesh, cfg->ny the global row count)
 * holds its rows plus ghost rows: one below and A above (A = 1 for the DG method, 2 for HDG,
 * whose first ghost row above is condensed and needs its own upper faces).  Every volume vector
 * has (rows + 1 + A) * nx cells in the usual cell-major layout, local row 0 and rows
 * rows+1..rows+A being the ghosts, and every trace vector the faces of those cells (x faces, then
 * y faces, each face owned by the cell below or left of it); dgh_slab_info gives where the
 * interior starts and its length.  The ghost rows and faces of vectors passed in belong to the
 * library: dgh_freeze, dgh_residual, dgh_admissible, dgh_dg_refresh, dgh_dg_apply, dgh_initial,
 * dgh_trace, dgh_hdg_refresh_projected (state and residual), dgh_hdg_retarget, dgh_hdg_apply,
 * dgh_hdg_recover and dgh_hdg_recovered_residual fill them from the neighbouring slabs (a halo
 * exchange of cell rows or face rows) before reading neighbours, and the residual, J*v, trace,
 * Schur apply and HDG right-hand-side outputs come back with zero ghosts.  Norms, integrals, L2 errors,
 * admissibility, the CFL rate, kernel status bits and the GMRES inner products are reduced over
 * all ranks, so every rank takes the same decisions (Newton, line search, GMRES restarts) and
 * receives the same scalars; every rank must make the same calls in the same order, each from
 * its own host thread or process.  Interior results equal the single-domain ones: residual,
 * J*v, frozen speeds, the CFL rate, the condensed right-hand side and the Schur apply on owned
 * faces bitwise; norms and the Newton update to rounding of the reduction order.  Covered: methods DG and HDG (HDG: at least two rows per rank), collocated
 * rule, block Jacobi, every precision and the FP32 condensation, BE and DIRK3 (dgh_integrator_*
 * on a slab context).  Not with slabs: method "both", over-integration, block ILU(0), J^T / the
 * adjoint, lockstep groups and graph-replayed GMRES cycles (refused).
 * Communicators (the communicator must outlive its contexts):
 *  - dgh_comm_nccl_create: one rank per process and GPU over NCCL; rank 0 makes the id with
 *    dgh_comm_nccl_unique_id and the host shares it (e.g. a torch.distributed broadcast).
 *    libnccl is resolved at run time (the copy already loaded, else DGH_NCCL_LIBRARY, else
 *    libnccl.so.2).
 *  - dgh_comm_local_create: `size` ranks inside one process (ranks[r] for rank r), each driven
 *    by its own host thread, on any devices (several slabs on one GPU included); collectives
 *    synchronise the ranks' streams and meet at host barriers, and a rank that waits longer
 *    than timeout_ms for its peers fails the group (DGH_ERR_COMM on every rank).
 *  - dgh_comm_fail: marks the group failed (a host that caught an error on one rank releases
 *    the others; a context failing with DGH_ERR_CUDA or DGH_ERR_COMM does this itself).
 *  - dgh_comm_set_timeout: how long a rank waits for its peers (local group: at a barrier,
 *    default the creation's timeout_ms, for the whole group; NCCL: for its stream, default
 *    300 s, after which the rank aborts its communicator, ending its own waiting NCCL kernels,
 *    and the call fails with DGH_ERR_COMM).  A rank that fails on its own therefore ends its
 *    peers' next collective with DGH_ERR_COMM in every kind.
 * dgh_comm_info: {rank, size, kind (0 local, 1 NCCL)}.  dgh_comm_error: the calling thread's
 * last dgh_comm_* failure. */
typedef struct dgh_comm dgh_comm;
int dgh_slab_rows(int ny, int size, int rank, int out[4]);
int dgh_comm_local_create(int size, int timeout_ms, dgh_comm **ranks);
int dgh_comm_nccl_unique_id(unsigned char id[128]);
int dgh_comm_nccl_create(const unsigned char id[128], int size, int rank, int device, dgh_comm **out);
int dgh_comm_info(const dgh_comm *comm, int out[3]);
int dgh_comm_fail(dgh_comm *comm, const char *why);
int dgh_comm_set_timeout(dgh_comm *comm, int timeout_ms);
/* The halo plan a slab context of mesh width nx, degree, `rows` interior rows and `above` ghost
 * rows above uses for volume vectors (trace = 0) or trace vectors (trace = 1): counts = the
 * number of regions sent to the rank below, sent to the rank above, received from the rank above
 * and received from the rank below; regions = their (offset, count) pairs in doubles, in that
 * order.  Host arithmetic only (no device). */
int dgh_slab_halo_plan(int nx, int degree, int rows, int above, int trace, int64_t regions[16], int counts[4]);
int dgh_comm_destroy(dgh_comm *comm);
const char *dgh_comm_error(void);
int dgh_ctx_create_slab(const dgh_config *cfg, dgh_comm *comm, dgh_ctx **out);
/* {global first row, interior rows, rank, size, first interior double of a volume vector,
 *  interior doubles, ghost rows above, doubles per face row of a trace vector} */
int dgh_slab_info(const dgh_ctx *ctx, int64_t out[8]);

/* ---- Discrete adjoint of the DG time integration (no counterpart in the reference) -------------
 * Objective J = sum over nodes of M rho^2 at the end of `steps` fixed steps (dt = cfl / rate of
 * each step's start state) of the context's integrator (SSP-DIRK3 or BE), DG method.  The
 * forward run records dt and the frozen wave speeds of every stage and checkpoints the state
 * every `checkpoint_every` steps; the reverse sweep recomputes each segment's stage states from
 * its checkpoint and solves J_s^T psi = Kbar_s per stage with GMRES on DGH_OP_DG_T.  dt and the
 * speeds are held fixed (the derivative of the recorded trajectory), and dgh_dirk3_replay
 * re-runs the forward model with exactly those values, for finite-difference checks.
 * host_grad receives dJ/dU(0) (size dgh_sizes()[0]). */
typedef struct dgh_adjoint_stats {
    double objective, final_time;
    int steps, checkpoints, forward_newton, adjoint_krylov, recomputed_steps;
} dgh_adjoint_stats;
int dgh_dirk3_adjoint(dgh_integrator *it, int steps, int checkpoint_every, const double *host_u0,
                      double *host_grad, dgh_adjoint_stats *stats);
int dgh_dirk3_replay(dgh_integrator *it, const double *host_u0, double *objective);

/* ---- Allocation-free residual ---------------------------------------------------------------
 * No counterpart in the reference.  R(u) as dgh_residual computes it on a context with the
 * collocated volume rule (quadrature 0 or degree+1; there is no quadrature argument), for callers that
 * cannot allocate device memory: an allocation-free time loop, work issued while a stream is
 * being captured into a CUDA graph (cudaMalloc is not permitted there), or a host that plans
 * every byte of device memory itself.  It needs no context and allocates nothing (no cudaMalloc,
 * no cudaFree, no allocating library call): its only scratch, the face restrictions of u
 * (16 (k+1) doubles per cell), lives in a fixed device array of DGH_NOALLOC_TRACE_CAPACITY
 * doubles (16 MiB) that every GPU loading this library holds until the process exits.
 *  - Limit: nx * ny * 16 * (degree + 1) <= DGH_NOALLOC_TRACE_CAPACITY (e.g. 120 x 120 cells at
 *    k = 8, 200 x 200 at k = 2); larger meshes return DGH_ERR_INVALID with the sizes in errbuf.
 *  - Inputs u, old (stage base) and speeds (frozen (a, b) per face node, as dgh_speeds returns
 *    them) and the output r are device pointers the caller owns; geometry follows testcase
 *    (DGH_TEST_*) and gamma = 3.  Work is queued on stream (a cudaStream_t; NULL = default).
 *  - The first call on a device looks up the scratch array's device address with that device
 *    current and keeps it; make that first call before any stream capture.  The kept address
 *    belongs to the device's primary context: after cudaDeviceReset (or anything else that
 *    destroys that context) it is stale, and the entry point must not be called again in
 *    that process.
 *  - Every call shares the one scratch array and the kernels overwrite all of it that they read,
 *    so nothing needs clearing between calls; but calls whose work overlaps on the GPU (other
 *    streams, other host threads) race on it and must be ordered by the caller.
 *  - errbuf (may be NULL) receives a message of at most errbuf_len bytes on failure. */
#define DGH_NOALLOC_TRACE_CAPACITY 2097152
int dgh_residual_noalloc(int nx, int ny, int degree, int testcase, double step_size, const double *u,
                         const double *old, const double *speeds, double *r, void *stream, char *errbuf,
                         int errbuf_len);

#ifdef __cplusplus
}
#endif
#endif /* DGH_GPU_H */
