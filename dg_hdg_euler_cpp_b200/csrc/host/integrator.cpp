// Host time integrator over the dgh_gpu.h C ABI: SSP-DIRK(4,3) or backward Euler, per-stage
// freezing, Newton with the residual-acceptance target, the HDG Schur-tolerance retry and the
// Armijo line search with the admissibility check (time_integrator.cpp:48-213).  Only scalars
// live on the host; every vector stays in device memory.
#include "dgh_gpu.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

namespace {
struct Failure {
    int code;
    std::string message;
};
}  // namespace

struct dgh_integrator {
    dgh_ctx *ctx = nullptr;
    int method = DGH_METHOD_DG;
    dgh_config cfg{};
    int64_t N = 0, NT = 0;
    double lx = 0, ly = 0;
    std::string err;
    std::vector<double *> owned;
    double *state = nullptr, *trial = nullptr, *residual = nullptr, *trial_residual = nullptr, *direction = nullptr;
    double *rhs = nullptr, *lambda = nullptr, *tdir = nullptr, *eq_err = nullptr, *indep = nullptr;
    double *step_state = nullptr, *stage_base = nullptr, *slopes[4] = {nullptr, nullptr, nullptr, nullptr};
    double *solution = nullptr;
    // current stage
    double tau = 0, old_norm = 0, initial_rms = -1, step = 0, rate = 0, elapsed_time = 0;
    int stage = 0, steps_done = 0, stages = 1;
    bool residual_ready = false;
    dgh_run_stats run{};
    // the reference's fixed limits (time_integrator.cpp:130,165): Schur attempts, line-search halvings
    int hdg_attempts = 4, line_search = 30;
    // discrete adjoint: recorded trajectory (dt per step, frozen speeds per stage, checkpoints)
    struct Adjoint {
        int steps = 0, every = 0, stages = 0;
        int64_t sz = 0;  // doubles of one speeds record
        std::vector<double> dt;
        double *speeds = nullptr;           // [steps][stages][sz]
        std::vector<double *> checkpoints;  // U^n for n % every == 0
        std::vector<double *> stage_states; // [every][stages]
        double *ubar = nullptr, *ubs = nullptr, *psi = nullptr, *kbar[4] = {nullptr, nullptr, nullptr, nullptr};
        double *u = nullptr, *step = nullptr;
        int forward_newton = 0, adjoint_krylov = 0, recomputed = 0;
    } adj;

    void ck(int rc) {
        if (rc != DGH_OK) throw Failure{rc, dgh_last_error(ctx)};
    }
    double *vec(int64_t n) {
        double *p = nullptr;
        ck(dgh_vec_alloc(ctx, n, &p));
        owned.push_back(p);
        return p;
    }
    double dual(const double *x) {
        double v = 0;
        ck(dgh_dual_norm(ctx, x, &v));
        return v;
    }
    double snorm(const double *x) {
        double v = 0;
        ck(dgh_state_norm(ctx, x, &v));
        return v;
    }
    // Residual (when not already available) and its norm at the top of a Newton iteration.
    double prepare(double &rms) {
        if (!residual_ready) ck(dgh_residual(ctx, state, residual));
        const double norm = dual(residual);
        rms = norm / std::sqrt(lx * ly);
        if (initial_rms < 0) initial_rms = rms;
        return norm;
    }
    // The body of one Newton iteration after the convergence test (time_integrator.cpp:104-220).
    void update(double norm, double rms, int it, dgh_update_stats &out) {
        const auto start = std::chrono::steady_clock::now();
        (void)start;
        const double allowance =
            128 * std::numeric_limits<double>::epsilon() * ((snorm(state) + old_norm) / tau + norm);
        const double target = std::max(10 * cfg.linear_tolerance * norm, allowance);
        // With dgh_config.forcing = 1 the linear solves stop at an absolute floor below which no
        // later test can see the difference: half the round-off allowance of the acceptance
        // target, and a tenth of the nonlinear tolerance in the same norm (so the Newton loop's
        // own convergence test is unaffected).  forcing = 0 keeps the reference's relative ltol.
        const double floor_abs =
            cfg.forcing ? std::min(.5 * allowance,
                                   .1 * cfg.nonlinear_tolerance * std::max(1., initial_rms) * std::sqrt(lx * ly))
                        : 0.;
        const double gmres_tol = norm > 0 ? std::max(cfg.linear_tolerance, floor_abs / norm) : cfg.linear_tolerance;
        int iterations = 0;
        double relative = 0;
        if (method == DGH_METHOD_DG) {
            ck(dgh_dg_refresh(ctx, state));
            ck(dgh_axpby(ctx, -1., residual, 0., residual, rhs, N));
            ck(dgh_block_jacobi_refresh(ctx, DGH_OP_DG));
            ck(dgh_gmres(ctx, DGH_OP_DG, rhs, direction, cfg.max_linear, gmres_tol, &iterations, &relative));
            const double *res = dgh_gmres_residual(ctx, DGH_OP_DG);
            ck(dgh_axpby(ctx, -1., res, 0., res, eq_err, N));
        } else if (cfg.condense32) {
            // FP32 condensation: the condensed system approximates the DG linearisation to FP32
            // accuracy, so J du = -r is solved by iterative refinement in FP64.  Each pass solves
            // the Schur system for the current DG residual, recovers the correction with the kept
            // FP32 cell factors, adds it, and forms the true residual e = J du + r with the FP64
            // J*v; the next pass retargets the condensation to e.  The passes stop once e is as
            // small as the FP64 solve's GMRES leaves it (ltol |r|, or the forcing floor), which is
            // below the acceptance target.  A pass's Schur tolerance goes no lower than the
            // estimated FP32 floor of one pass (below it GMRES iterations buy nothing) nor than
            // what the stop still needs.
            const double stop = std::max(cfg.linear_tolerance * norm, floor_abs);
            ck(dgh_hdg_refresh_projected(ctx, state, residual));
            ck(dgh_hdg_rhs(ctx, rhs));
            ck(dgh_block_jacobi_refresh(ctx, DGH_OP_HDG));
            double floor_est = 1e-6, current = norm;
            bool valid = false;
            for (int pass = 0; pass < 2 * hdg_attempts && !valid; ++pass) {
                const double tolerance = std::max({cfg.linear_tolerance, floor_est, .3 * stop / current});
                int cur = 0;
                double rel = 0;
                ck(dgh_gmres(ctx, DGH_OP_HDG, rhs, tdir, cfg.max_linear, tolerance, &cur, &rel));
                iterations += cur;
                relative = rel;
                ck(dgh_hdg_recover(ctx, tdir, pass == 0 ? direction : indep));
                if (pass > 0) ck(dgh_axpby(ctx, 1., direction, 1., indep, direction, N));
                ck(dgh_dg_apply(ctx, direction, eq_err));
                ck(dgh_axpby(ctx, 1., eq_err, 1., residual, eq_err, N));
                const double next = dual(eq_err);
                if (next <= stop) {
                    valid = true;
                } else {
                    const double achieved = next / current;
                    if (achieved > 10 * tolerance) floor_est = std::min(.1, achieved);
                    current = next;
                    ck(dgh_hdg_retarget(ctx, eq_err));
                    ck(dgh_hdg_rhs(ctx, rhs));
                }
            }
            if (!valid) throw Failure{DGH_ERR_SOLVER, "Recovered DG residual criterion failed after Schur refinement"};
        } else {
            ck(dgh_hdg_refresh_projected(ctx, state, residual));
            ck(dgh_hdg_rhs(ctx, rhs));
            ck(dgh_block_jacobi_refresh(ctx, DGH_OP_HDG));
            double tolerance = gmres_tol;
            bool valid = false;
            for (int attempt = 0; attempt < hdg_attempts; ++attempt) {
                int cur = 0;
                double rel = 0;
                ck(dgh_gmres(ctx, DGH_OP_HDG, rhs, tdir, cfg.max_linear, tolerance, &cur, &rel));
                iterations += cur;
                relative = rel;
                ck(dgh_hdg_recover(ctx, tdir, direction));
                const double *res = dgh_gmres_residual(ctx, DGH_OP_HDG);
                ck(dgh_axpby(ctx, -1., res, 0., res, lambda, NT));
                ck(dgh_hdg_recovered_residual(ctx, lambda, eq_err));
                valid = dual(eq_err) <= target;
                if (valid) break;
                tolerance *= .01;
            }
            if (!valid) throw Failure{DGH_ERR_SOLVER, "Recovered DG residual criterion failed after Schur refinement"};
        }
        const double error_norm = dual(eq_err);
        if (!(error_norm <= target)) throw Failure{DGH_ERR_SOLVER, "DG Newton linear residual too large"};
        if (method == DGH_METHOD_HDG && cfg.check_update) {
            // time_integrator.cpp:153-162: an independent DG J*v of the recovered update.  The
            // condensation linearised the same state, so the DG caches are already current.
            ck(dgh_dg_apply(ctx, direction, indep));
            ck(dgh_axpby(ctx, 1., indep, 1., residual, indep, N));
            if (!(dual(indep) <= std::max(4 * target, 1e-12)))
                throw Failure{DGH_ERR_SOLVER, "Independent recovered DG equation check failed"};
            ck(dgh_axpby(ctx, 1., indep, -1., eq_err, indep, N));
            if (!(dual(indep) <= std::max(4 * allowance, 1e-12)))
                throw Failure{DGH_ERR_SOLVER, "Recovered residual identity failed"};
        }
        double damping = 1.;
        bool accepted = false;
        for (int search = 0; search < line_search; ++search) {
            ck(dgh_axpby(ctx, 1., state, damping, direction, trial, N));
            int ok = 0;
            ck(dgh_admissible(ctx, trial, &ok));
            if (ok) {
                ck(dgh_residual(ctx, trial, trial_residual));
                if (dual(trial_residual) <= (1 - 1e-4 * damping) * norm + allowance) {
                    accepted = true;
                    break;
                }
            }
            damping *= .5;
        }
        if (!accepted) throw Failure{DGH_ERR_SOLVER, "Newton line search failed"};
        std::swap(state, trial);
        std::swap(residual, trial_residual);
        residual_ready = true;
        out.step = steps_done;
        out.stage = stage;
        out.iteration = it;
        out.krylov_iterations = iterations;
        out.linear_relative_residual = relative;
        out.dg_linear_relative_residual = norm > 0 ? error_norm / norm : 0.;
        out.residual_physical_rms = rms;
        out.damping = damping;
    }
};

namespace {
constexpr double kAlpha = .24169426078821, kBeta = kAlpha / 4., kEta = .12915286960590;
constexpr double kA[4][4] = {{kAlpha, 0, 0, 0}, {-kAlpha, kAlpha, 0, 0}, {0, 1 - kAlpha, kAlpha, 0},
                             {kBeta, kEta, .5 - kBeta - kEta - kAlpha, kAlpha}};
constexpr double kB[4] = {0, 1. / 6, 1. / 6, 2. / 3}, kC[4] = {kAlpha, 0, 1, .5};
using Clock = std::chrono::steady_clock;
double since(Clock::time_point s) { return std::chrono::duration<double>(Clock::now() - s).count(); }

template <class F> int guarded(dgh_integrator *it, F &&f) {
    if (!it) return DGH_ERR_INVALID;
    try {
        f();
        return DGH_OK;
    } catch (const Failure &e) {
        it->err = e.message;
        return e.code;
    }
}
}  // namespace

extern "C" {

const char *dgh_integrator_error(const dgh_integrator *it) { return it ? it->err.c_str() : ""; }

int dgh_integrator_create(dgh_ctx *ctx, int method, dgh_integrator **out) {
    if (!ctx || !out || (method != DGH_METHOD_DG && method != DGH_METHOD_HDG)) return DGH_ERR_INVALID;
    auto *it = new dgh_integrator;
    it->ctx = ctx;
    it->method = method;
    const int rc = guarded(it, [&] {
        int64_t s[8];
        it->ck(dgh_sizes(ctx, s));
        it->N = s[0];
        it->NT = s[1];
        double geo[4];
        it->ck(dgh_geometry(ctx, geo));
        it->lx = geo[2];
        it->ly = geo[3];
        it->ck(dgh_get_config(ctx, &it->cfg));
        const int64_t N = it->N, NT = it->NT;
        it->state = it->vec(N); it->trial = it->vec(N); it->residual = it->vec(N);
        it->trial_residual = it->vec(N); it->direction = it->vec(N);
        it->rhs = it->vec(method == DGH_METHOD_DG ? N : NT);
        it->lambda = it->vec(NT); it->tdir = it->vec(NT);
        it->eq_err = it->vec(N); it->indep = it->vec(N);
        it->step_state = it->vec(N); it->stage_base = it->vec(N); it->solution = it->vec(N);
        for (auto &p : it->slopes) p = it->vec(N);
    });
    if (rc != DGH_OK) {
        dgh_integrator_destroy(it);
        return rc;
    }
    *out = it;
    return DGH_OK;
}

int dgh_integrator_destroy(dgh_integrator *it) {
    if (!it) return DGH_OK;
    for (double *p : it->owned) dgh_vec_free(it->ctx, p);
    delete it;
    return DGH_OK;
}

double *dgh_integrator_state(dgh_integrator *it) { return it ? it->state : nullptr; }

int dgh_integrator_set_limits(dgh_integrator *it, int hdg_attempts, int line_search) {
    if (!it || hdg_attempts < 0 || line_search < 0) return DGH_ERR_INVALID;
    it->hdg_attempts = hdg_attempts;
    it->line_search = line_search;
    return DGH_OK;
}

// time_integrator.cpp:48-213 (the full run).  The integrator reads its configuration from the
// context it was created on.
int dgh_advance(dgh_integrator *it, double *host_solution, dgh_run_stats *stats, dgh_update_stats *updates,
                int max_updates) {
    return guarded(it, [&] {
        const dgh_config &c = it->cfg;
        dgh_ctx *ctx = it->ctx;
        const int64_t N = it->N;
        it->ck(dgh_upload(ctx, it->solution, host_solution, N));
        int ok = 0;
        it->ck(dgh_admissible(ctx, it->solution, &ok));
        if (!ok) throw Failure{DGH_ERR_STATE, "Invalid initial solution"};
        const double shock = c.testcase == DGH_TEST_WAVE ? std::numeric_limits<double>::infinity()
                                                         : 4 / ((3. + 1) * std::acos(-1.));
        if (!(c.steps > 0 || c.final_time < shock)) throw Failure{DGH_ERR_STATE, "Final time reaches simple-wave shock"};
        const int stages = c.integrator == DGH_INTEGRATOR_BE ? 1 : 4;
        it->stages = stages;
        dgh_run_stats st{};
        int recorded = 0;
        double rate0 = 0;
        it->ck(dgh_freeze(ctx, it->solution, &rate0));
        double initial_integral[4];
        it->ck(dgh_integral(ctx, it->solution, initial_integral));
        const auto begin = Clock::now();
        it->steps_done = 0;
        while (c.steps > 0 ? st.steps < c.steps : st.final_time < c.final_time) {
            double rate = 0;
            it->ck(dgh_freeze(ctx, it->solution, &rate));
            double step = c.cfl / rate;
            if (c.steps == 0) {
                const double remaining = c.final_time - st.final_time;
                step = std::min(step, remaining);
                if (remaining - step <= 16 * std::numeric_limits<double>::epsilon() * std::max(remaining, c.final_time))
                    step = remaining;
            }
            if (!(std::isfinite(step) && step > 0 && st.final_time + step > st.final_time))
                throw Failure{DGH_ERR_STATE, "Invalid CFL step"};
            if (!(st.final_time + step < shock)) throw Failure{DGH_ERR_STATE, "Step reaches simple-wave shock"};
            it->ck(dgh_axpby(ctx, 1., it->solution, 0., it->solution, it->step_state, N));
            it->ck(dgh_axpby(ctx, 1., it->solution, 0., it->solution, it->state, N));
            for (int stage = 0; stage < stages; ++stage) {
                const double diagonal = stages == 1 ? 1. : kA[stage][stage];
                it->ck(dgh_axpby(ctx, 1., it->step_state, 0., it->step_state, it->stage_base, N));
                for (int j = 0; j < stage; ++j)
                    it->ck(dgh_axpby(ctx, 1., it->stage_base, step * kA[stage][j], it->slopes[j], it->stage_base, N));
                double unused = 0;
                if (stage > 0) it->ck(dgh_freeze(ctx, it->state, &unused));
                it->ck(dgh_set_stage(ctx, it->stage_base, diagonal * step));
                it->tau = diagonal * step;
                it->old_norm = it->snorm(it->stage_base);
                it->stage = stage;
                it->initial_rms = -1.;
                it->residual_ready = false;
                const int limit = c.newton_steps > 0 ? c.newton_steps : c.max_newton;
                bool converged = false;
                for (int k = 0; k <= limit; ++k) {
                    const auto t0 = Clock::now();
                    double rms = 0;
                    const double norm = it->prepare(rms);
                    if (c.newton_steps == 0 && rms <= c.nonlinear_tolerance * std::max(1., it->initial_rms)) {
                        converged = true;
                        break;
                    }
                    if (k == limit) break;
                    dgh_update_stats u{};
                    it->steps_done = st.steps;
                    it->update(norm, rms, k, u);
                    const double duration = since(t0);
                    u.iteration_s = duration;
                    u.time = st.final_time + step;
                    u.stage_time = st.final_time + (stages == 1 ? 1. : kC[stage]) * step;
                    u.dt = step;
                    u.cfl = step * rate;
                    st.max_linear_residual = std::max(st.max_linear_residual, u.linear_relative_residual);
                    st.max_dg_linear_residual = std::max(st.max_dg_linear_residual, u.dg_linear_relative_residual);
                    st.krylov_iterations += u.krylov_iterations;
                    if (st.newton_iterations >= c.warmup_updates) {
                        st.measured_newton_seconds += duration;
                        ++st.measured_updates;
                    }
                    ++st.newton_iterations;
                    if (updates && recorded < max_updates) updates[recorded] = u;
                    ++recorded;
                }
                if (!(converged || c.newton_steps > 0)) throw Failure{DGH_ERR_SOLVER, "Newton iteration limit reached"};
                it->ck(dgh_axpby(ctx, 1. / it->tau, it->state, -1. / it->tau, it->stage_base, it->slopes[stage], N));
            }
            if (stages == 1) {
                it->ck(dgh_axpby(ctx, 1., it->state, 0., it->state, it->solution, N));
            } else {
                it->ck(dgh_axpby(ctx, 1., it->step_state, 0., it->step_state, it->solution, N));
                for (int s = 0; s < stages; ++s)
                    it->ck(dgh_axpby(ctx, 1., it->solution, step * kB[s], it->slopes[s], it->solution, N));
                int ok2 = 0;
                it->ck(dgh_admissible(ctx, it->solution, &ok2));
                if (!ok2) throw Failure{DGH_ERR_STATE, "DIRK3 step produced an inadmissible state"};
            }
            st.final_time = c.steps == 0 && step >= c.final_time - st.final_time ? c.final_time : st.final_time + step;
            st.minimum_step = st.steps == 0 ? step : std::min(st.minimum_step, step);
            st.maximum_step = std::max(st.maximum_step, step);
            ++st.steps;
            double now[4];
            it->ck(dgh_integral(ctx, it->solution, now));
            double drift = 0;
            for (int v = 0; v < 4; ++v) drift = std::max(drift, std::abs(now[v] - initial_integral[v]));
            st.conservation_drift = std::max(st.conservation_drift, drift);
        }
        st.seconds = since(begin);
        st.updates_recorded = recorded;
        it->ck(dgh_download(ctx, host_solution, it->solution, N));
        if (stats) *stats = st;
    });
}

int dgh_stage_begin(dgh_integrator *it, const double *u, double *dt) {
    return guarded(it, [&] {
        dgh_ctx *ctx = it->ctx;
        const int64_t N = it->N;
        double rate = 0;
        it->ck(dgh_freeze(ctx, u, &rate));
        const double step = it->cfg.cfl / rate;
        it->ck(dgh_axpby(ctx, 1., u, 0., u, it->state, N));
        it->ck(dgh_axpby(ctx, 1., u, 0., u, it->stage_base, N));
        it->ck(dgh_set_stage(ctx, it->stage_base, step));
        it->tau = step;
        it->step = step;
        it->rate = rate;
        it->old_norm = it->snorm(it->stage_base);
        it->stage = 0;
        it->initial_rms = -1.;
        it->residual_ready = false;
        if (dt) *dt = step;
    });
}

int dgh_newton_update(dgh_integrator *it, dgh_update_stats *stats) {
    return guarded(it, [&] {
        const auto t0 = Clock::now();
        double rms = 0;
        const double norm = it->prepare(rms);
        dgh_update_stats u{};
        it->update(norm, rms, 0, u);
        it->ck(dgh_sync(it->ctx));
        u.iteration_s = since(t0);
        u.dt = it->step;
        u.time = it->step;
        u.stage_time = it->step;
        u.cfl = it->step * it->rate;
        if (stats) *stats = u;
    });
}

int dgh_newton_update_host(dgh_integrator *it, double *host_state, dgh_update_stats *stats) {
    return guarded(it, [&] {
        const auto t0 = Clock::now();
        it->ck(dgh_upload(it->ctx, it->state, host_state, it->N));
        it->residual_ready = false;
        double rms = 0;
        const double norm = it->prepare(rms);
        dgh_update_stats u{};
        it->update(norm, rms, 0, u);
        it->ck(dgh_download(it->ctx, host_state, it->state, it->N));
        u.iteration_s = since(t0);
        u.dt = it->step;
        u.time = it->step;
        u.stage_time = it->step;
        u.cfl = it->step * it->rate;
        if (stats) *stats = u;
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Discrete adjoint of SSP-DIRK(4,3) (or backward Euler) for the DG solve, with the step sizes and
// the frozen wave speeds of the recorded forward trajectory held fixed (they are non-smooth
// functions of the state: dt = CFL / max(...), Einfeldt bounds with max()).  For stage s,
// R(U_s) = M (U_s - U_b,s)/tau_s - L(U_s) = 0 and K_s = (U_s - U_b,s)/tau_s, so with
// psi = J_s^{-T} Kbar_s the stage base receives Ubar_b,s = (M psi / tau_s - Kbar_s) / tau_s, where
// Kbar_s = dt b_s Ubar^{n+1} + sum_{r>s} dt a_rs Ubar_b,r and Ubar^n = Ubar^{n+1} + sum_s Ubar_b,s.
// J_s^T solves use GMRES on the adjoint operator with the transposed block-Jacobi factors.
namespace {
// One stage's Newton solve to the nonlinear tolerance (time_integrator.cpp:133-142 without the
// statistics); returns the number of updates.
int newton_stage(dgh_integrator *it) {
    const dgh_config &c = it->cfg;
    it->initial_rms = -1.;
    it->residual_ready = false;
    int updates = 0;
    for (int k = 0; k <= c.max_newton; ++k) {
        double rms = 0;
        const double norm = it->prepare(rms);
        if (rms <= c.nonlinear_tolerance * std::max(1., it->initial_rms)) return updates;
        if (k == c.max_newton) break;
        dgh_update_stats u{};
        it->update(norm, rms, k, u);
        ++updates;
    }
    throw Failure{DGH_ERR_SOLVER, "Newton iteration limit reached"};
}

// Forward DIRK3/BE from `u` over steps [first, last): records dt and speeds when `record`,
// replays them otherwise; stores stage solutions into adj.stage_states when `keep`.
void forward(dgh_integrator *it, double *u, int first, int last, bool record, bool keep, bool checkpoint) {
    auto &a = it->adj;
    dgh_ctx *ctx = it->ctx;
    const int64_t N = it->N;
    const int S = a.stages;
    for (int n = first; n < last; ++n) {
        if (checkpoint && n % a.every == 0) it->ck(dgh_axpby(ctx, 1., u, 0., u, a.checkpoints[n / a.every], N));
        double dt;
        if (record) {
            double rate = 0;
            it->ck(dgh_freeze(ctx, u, &rate));
            dt = it->cfg.cfl / rate;
            a.dt[n] = dt;
            it->ck(dgh_copy_speeds(ctx, a.speeds + ((size_t)n * S) * a.sz));
        } else {
            dt = a.dt[n];
            it->ck(dgh_set_speeds(ctx, a.speeds + ((size_t)n * S) * a.sz));
        }
        it->ck(dgh_axpby(ctx, 1., u, 0., u, it->step_state, N));
        it->ck(dgh_axpby(ctx, 1., u, 0., u, it->state, N));
        for (int s = 0; s < S; ++s) {
            const double diag = S == 1 ? 1. : kA[s][s];
            it->ck(dgh_axpby(ctx, 1., it->step_state, 0., it->step_state, it->stage_base, N));
            for (int j = 0; j < s; ++j)
                it->ck(dgh_axpby(ctx, 1., it->stage_base, dt * kA[s][j], it->slopes[j], it->stage_base, N));
            if (s > 0) {
                if (record) {
                    double unused = 0;
                    it->ck(dgh_freeze(ctx, it->state, &unused));
                    it->ck(dgh_copy_speeds(ctx, a.speeds + ((size_t)n * S + s) * a.sz));
                } else {
                    it->ck(dgh_set_speeds(ctx, a.speeds + ((size_t)n * S + s) * a.sz));
                }
            }
            it->ck(dgh_set_stage(ctx, it->stage_base, diag * dt));
            it->tau = diag * dt;
            it->old_norm = it->snorm(it->stage_base);
            a.forward_newton += newton_stage(it);
            if (keep) it->ck(dgh_axpby(ctx, 1., it->state, 0., it->state, a.stage_states[(n - first) * S + s], N));
            it->ck(dgh_axpby(ctx, 1. / it->tau, it->state, -1. / it->tau, it->stage_base, it->slopes[s], N));
        }
        it->ck(dgh_axpby(ctx, 1., it->step_state, 0., it->step_state, u, N));
        for (int s = 0; s < S; ++s) {
            const double bs = S == 1 ? 1. : kB[s];
            it->ck(dgh_axpby(ctx, 1., u, dt * bs, it->slopes[s], u, N));
        }
    }
}

void prepare_adjoint(dgh_integrator *it, int steps, int every) {
    auto &a = it->adj;
    if (a.steps == steps && a.every == every && a.speeds) return;
    int64_t s8[8];
    it->ck(dgh_sizes(it->ctx, s8));
    a.steps = steps;
    a.every = every;
    a.stages = it->cfg.integrator == DGH_INTEGRATOR_BE ? 1 : 4;
    a.sz = 2 * s8[4] * s8[5];
    a.dt.assign(steps, 0.);
    a.speeds = it->vec((int64_t)steps * a.stages * a.sz);
    a.checkpoints.clear();
    for (int k = 0; k < (steps + every - 1) / every; ++k) a.checkpoints.push_back(it->vec(it->N));
    a.stage_states.clear();
    for (int k = 0; k < every * a.stages; ++k) a.stage_states.push_back(it->vec(it->N));
    a.ubar = it->vec(it->N);
    a.ubs = it->vec(it->N);
    a.psi = it->vec(it->N);
    for (auto &p : a.kbar) p = it->vec(it->N);
    a.u = it->vec(it->N);
    a.step = it->vec(it->N);
}
}  // namespace

extern "C" {
int dgh_dirk3_adjoint(dgh_integrator *it, int steps, int checkpoint_every, const double *host_u0, double *host_grad,
                      dgh_adjoint_stats *stats) {
    return guarded(it, [&] {
        if (it->method != DGH_METHOD_DG) throw Failure{DGH_ERR_INVALID, "The discrete adjoint runs on the DG operator"};
        if (steps <= 0 || checkpoint_every <= 0) throw Failure{DGH_ERR_INVALID, "Invalid step or checkpoint count"};
        prepare_adjoint(it, steps, checkpoint_every);
        auto &a = it->adj;
        dgh_ctx *ctx = it->ctx;
        const int64_t N = it->N;
        const int S = a.stages;
        a.forward_newton = a.adjoint_krylov = a.recomputed = 0;
        it->ck(dgh_upload(ctx, a.u, host_u0, N));
        forward(it, a.u, 0, steps, true, false, true);
        double objective = 0;
        it->ck(dgh_rho2(ctx, a.u, &objective, a.ubar));
        double final_time = 0;
        for (double d : a.dt) final_time += d;
        const int segments = (steps + checkpoint_every - 1) / checkpoint_every;
        for (int seg = segments - 1; seg >= 0; --seg) {
            const int c0 = seg * checkpoint_every, c1 = std::min(steps, c0 + checkpoint_every);
            it->ck(dgh_axpby(ctx, 1., a.checkpoints[seg], 0., a.checkpoints[seg], a.step, N));
            forward(it, a.step, c0, c1, false, true, false);  // recompute the segment's stage states
            a.recomputed += c1 - c0;
            for (int n = c1 - 1; n >= c0; --n) {
                const double dt = a.dt[n];
                for (int s = 0; s < S; ++s) {
                    const double bs = S == 1 ? 1. : kB[s];
                    it->ck(dgh_axpby(ctx, dt * bs, a.ubar, 0., a.ubar, a.kbar[s], N));
                }
                for (int s = S - 1; s >= 0; --s) {
                    const double tau = (S == 1 ? 1. : kA[s][s]) * dt;
                    double *us = a.stage_states[(n - c0) * S + s];
                    it->ck(dgh_set_speeds(ctx, a.speeds + ((size_t)n * S + s) * a.sz));
                    it->ck(dgh_set_stage(ctx, us, tau));
                    it->ck(dgh_dg_refresh(ctx, us));
                    it->ck(dgh_block_jacobi_refresh(ctx, DGH_OP_DG));
                    int iters = 0;
                    double rel = 0;
                    it->ck(dgh_gmres(ctx, DGH_OP_DG_T, a.kbar[s], a.psi, it->cfg.max_linear, it->cfg.linear_tolerance,
                                     &iters, &rel));
                    a.adjoint_krylov += iters;
                    it->ck(dgh_mass_axpby(ctx, 1. / (tau * tau), a.psi, -1. / tau, a.kbar[s], a.ubs));
                    it->ck(dgh_axpby(ctx, 1., a.ubar, 1., a.ubs, a.ubar, N));
                    for (int j = 0; j < s; ++j)
                        it->ck(dgh_axpby(ctx, 1., a.kbar[j], dt * kA[s][j], a.ubs, a.kbar[j], N));
                }
            }
        }
        it->ck(dgh_download(ctx, host_grad, a.ubar, N));
        if (stats) {
            stats->objective = objective;
            stats->final_time = final_time;
            stats->steps = steps;
            stats->checkpoints = segments;
            stats->forward_newton = a.forward_newton;
            stats->adjoint_krylov = a.adjoint_krylov;
            stats->recomputed_steps = a.recomputed;
        }
    });
}

int dgh_dirk3_replay(dgh_integrator *it, const double *host_u0, double *objective) {
    return guarded(it, [&] {
        auto &a = it->adj;
        if (!a.speeds) throw Failure{DGH_ERR_INVALID, "Run dgh_dirk3_adjoint first to record a trajectory"};
        it->ck(dgh_upload(it->ctx, a.u, host_u0, it->N));
        forward(it, a.u, 0, a.steps, false, false, false);
        it->ck(dgh_rho2(it->ctx, a.u, objective, nullptr));
    });
}
}  // extern "C"
