// Test infrastructure only: C entry points of the CPU oracle, loaded by tests/ through ctypes.
// Each function mirrors one call of the reference's solver surface (dg_hdg_2d/include/euler/*).
// Functions return 0 on success and 1 on a thrown require(); oracle_error() gives the text.
#include "dgh_oracle.hpp"

#include <map>

#include <cstring>
#include <memory>
#include <sstream>

using namespace oracle;

namespace {
thread_local std::string last_error;
struct Handle {
    std::unique_ptr<Problem> p;
    std::unique_ptr<DGOperator> dg;
    std::unique_ptr<HybridOperator> hdg;
    std::unique_ptr<BlockJacobi> pc_dg, pc_hdg;
    std::unique_ptr<BlockILU0> ilu_dg;  // 2D block ILU(0) on the cartesian block graph (no reference counterpart)
    Vec residual;
};
template <class F> int guard(F &&f) {
    try {
        f();
        return 0;
    } catch (const std::exception &e) {
        last_error = e.what();
        return 1;
    }
}
Config config_from(const char *args) {
    std::istringstream in(args ? args : "");
    std::vector<std::string> words{"oracle"};
    for (std::string w; in >> w;) words.push_back(w);
    std::vector<char *> argv;
    for (auto &w : words) argv.push_back(w.data());
    return parse((int)argv.size(), argv.data());
}
Vec vec(const double *p, size_t n) { return Vec(p, p + n); }
void out(const Vec &v, double *p) { std::memcpy(p, v.data(), v.size() * sizeof(double)); }
}  // namespace

extern "C" {
const char *oracle_error() { return last_error.c_str(); }
void oracle_set_error(const char *m) { last_error = m; }
void oracle_set_threads(int t) { set_threads(t); }
int oracle_run(int argc, char **argv) { return run_main(argc, argv); }

void *oracle_create(const char *args) {
    Handle *h = nullptr;
    if (guard([&] {
            auto c = config_from(args);
            h = new Handle;
            h->p = std::make_unique<Problem>(c);
            h->dg = std::make_unique<DGOperator>(*h->p);
            h->hdg = std::make_unique<HybridOperator>(*h->p);
        }))
        return nullptr;
    return h;
}
void oracle_destroy(void *h) { delete static_cast<Handle *>(h); }
// sizes: volume size, trace size, block width, cells, faces, nodes per direction
int oracle_sizes(void *hv, long long *s) {
    auto *h = static_cast<Handle *>(hv);
    s[0] = h->p->size(); s[1] = h->p->trace_size(); s[2] = h->p->block;
    s[3] = h->p->cells; s[4] = h->p->face_count(); s[5] = h->p->n;
    return 0;
}
int oracle_geometry(void *hv, double *g) {  // hx, hy, lx, ly
    auto *h = static_cast<Handle *>(hv);
    g[0] = h->p->hx; g[1] = h->p->hy; g[2] = h->p->example.lx; g[3] = h->p->example.ly;
    return 0;
}
int oracle_basis(void *hv, double *x, double *w) {
    auto *h = static_cast<Handle *>(hv);
    out(h->p->basis.x, x); out(h->p->basis.w, w);
    return 0;
}
int oracle_mass(void *hv, double *m, double *tm) {
    auto *h = static_cast<Handle *>(hv);
    out(h->p->mass, m); out(h->p->trace_mass, tm);
    return 0;
}
int oracle_initial(void *hv, double *u) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] { Vec v; h->p->initial(v); out(v, u); });
}
int oracle_exact(void *hv, double x, double y, double t, double *s) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] { State e = h->p->example.exact(x, y, t); for (int v = 0; v < 4; ++v) s[v] = e[v]; });
}
int oracle_freeze(void *hv, const double *u, double *rate) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] { *rate = h->p->freeze(vec(u, h->p->size())); });
}
int oracle_speeds(void *hv, double *ab) {
    auto *h = static_cast<Handle *>(hv);
    for (size_t i = 0; i < h->p->speeds.size(); ++i) { ab[2 * i] = h->p->speeds[i].a; ab[2 * i + 1] = h->p->speeds[i].b; }
    return 0;
}
int oracle_set_stage(void *hv, const double *old, double step) {
    auto *h = static_cast<Handle *>(hv);
    h->p->old = vec(old, h->p->size());
    h->p->step_size = step;
    return 0;
}
int oracle_residual(void *hv, const double *u, double *r) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] { Vec o; h->p->dg_residual(vec(u, h->p->size()), o); out(o, r); });
}
int oracle_trace(void *hv, const double *u, double *lam) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] { Vec o; h->p->trace(vec(u, h->p->size()), o); out(o, lam); });
}
int oracle_hybrid_residual(void *hv, const double *u, const double *lam, double *r, double *g) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] {
        Vec ro, go;
        h->p->hybrid_residual(vec(u, h->p->size()), vec(lam, h->p->trace_size()), ro, go);
        out(ro, r); out(go, g);
    });
}
int oracle_admissible(void *hv, const double *u, int *ok) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] { *ok = h->p->admissible(vec(u, h->p->size())) ? 1 : 0; });
}
int oracle_integral(void *hv, const double *u, double *s) {
    auto *h = static_cast<Handle *>(hv);
    State i = h->p->integral(vec(u, h->p->size()));
    for (int v = 0; v < 4; ++v) s[v] = i[v];
    return 0;
}
int oracle_l2_error(void *hv, const double *u, double t, double *s) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] { State e = h->p->error(vec(u, h->p->size()), t); for (int v = 0; v < 4; ++v) s[v] = e[v]; });
}
int oracle_dg_refresh(void *hv, const double *u) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] { h->dg->refresh(vec(u, h->p->size())); });
}
int oracle_dg_apply(void *hv, const double *d, double *o) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] { Vec r; h->dg->apply(vec(d, h->p->size()), r); out(r, o); });
}
int oracle_dg_apply_transpose(void *hv, const double *w, double *o) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] { Vec r; h->dg->apply_transpose(vec(w, h->p->size()), r); out(r, o); });
}
int oracle_dg_block(void *hv, int row, int col, double *o) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] { h->dg->block(row, col, o); });
}
int oracle_trace_diagonal(void *hv, double *o) {
    auto *h = static_cast<Handle *>(hv);
    out(h->dg->trace_diagonal(), o);
    return 0;
}
int oracle_dg_precond_refresh(void *hv) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] {
        h->pc_dg = std::make_unique<BlockJacobi>(h->p->cells, h->p->block);
        h->pc_dg->refresh([&](int r, int c, double *o) { h->dg->block(r, c, o); });
    });
}
int oracle_dg_precond_apply(void *hv, const double *x, double *z) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] { Vec o; h->pc_dg->apply(vec(x, h->p->size()), o); out(o, z); });
}
int oracle_hdg_refresh(void *hv, const double *u, const double *r) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] { h->hdg->refresh_projected(vec(u, h->p->size()), vec(r, h->p->size())); });
}
int oracle_hdg_rhs(void *hv, double *o) {
    auto *h = static_cast<Handle *>(hv);
    out(h->hdg->rhs(), o);
    return 0;
}
int oracle_hdg_apply(void *hv, const double *d, double *o) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] { Vec r; h->hdg->apply(vec(d, h->p->trace_size()), r); out(r, o); });
}
int oracle_hdg_block(void *hv, int row, int col, double *o) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] { h->hdg->block(row, col, o); });
}
int oracle_hdg_recover(void *hv, const double *d, double *o) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] { Vec r; h->hdg->recover(vec(d, h->p->trace_size()), r); out(r, o); });
}
int oracle_hdg_recovered_residual(void *hv, const double *e, double *o) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] { Vec r; h->hdg->recovered_residual_from_schur(vec(e, h->p->trace_size()), r); out(r, o); });
}
int oracle_hdg_schur(void *hv, double *o) {  // [cell][t x t] column-major
    auto *h = static_cast<Handle *>(hv);
    out(h->hdg->schur(), o);
    return 0;
}
int oracle_hdg_precond_refresh(void *hv) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] {
        h->pc_hdg = std::make_unique<BlockJacobi>(h->p->face_count(), h->p->face_width());
        h->pc_hdg->refresh([&](int r, int c, double *o) { h->hdg->block(r, c, o); });
    });
}
int oracle_hdg_precond_apply(void *hv, const double *x, double *z) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] { Vec o; h->pc_hdg->apply(vec(x, h->p->trace_size()), o); out(o, z); });
}
// Block ILU(0) of the DG Jacobian in the natural ordering on BlockGraph::cartesian, the pattern
// the reference's direct solver assembles in 2D (time_integrator.cpp:35); the reference's 2D
// front end accepts block-jacobi only (config.cpp:102), so this exists to measure what ILU(0)
// would save in 2D.
int oracle_dg_precond_refresh_ilu(void *hv) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] {
        h->ilu_dg = std::make_unique<BlockILU0>(cartesian_adjacency(h->p->nx, h->p->ny), h->p->block);
        h->ilu_dg->refresh([&](int r, int c, double *o) { h->dg->block(r, c, o); });
    });
}
// op 0: DG Jv with block-Jacobi; op 1: Schur apply with face block-Jacobi; op 2: DG Jv with the
// z = M^{-1} x with the 2D block ILU(0) factors of oracle_dg_precond_refresh_ilu
int oracle_dg_precond_apply_ilu(void *hv, const double *x, double *z) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] { Vec o; h->ilu_dg->apply(vec(x, h->p->size()), o); out(o, z); });
}
// 2D block ILU(0) of oracle_dg_precond_refresh_ilu
int oracle_gmres(void *hv, int op, int restart, const double *rhs, double *x, int limit, double tol,
                 int *iters, double *rel, double *residual) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] {
        const int n = op != 1 ? h->p->size() : h->p->trace_size();
        GMRES g(n, restart, op != 1 ? h->p->inverse_mass : h->p->inverse_trace_mass);
        Vec xv;
        LinearResult res;
        if (op == 0)
            res = g.solve(Action{h->dg.get(), [](const void *c, const Vec &a, Vec &b) { static_cast<const DGOperator *>(c)->apply(a, b); }},
                          Action{h->pc_dg.get(), [](const void *c, const Vec &a, Vec &b) { static_cast<const BlockJacobi *>(c)->apply(a, b); }},
                          vec(rhs, n), xv, limit, tol);
        else if (op == 2)
            res = g.solve(Action{h->dg.get(), [](const void *c, const Vec &a, Vec &b) { static_cast<const DGOperator *>(c)->apply(a, b); }},
                          Action{h->ilu_dg.get(), [](const void *c, const Vec &a, Vec &b) { static_cast<const BlockILU0 *>(c)->apply(a, b); }},
                          vec(rhs, n), xv, limit, tol);
        else
            res = g.solve(Action{h->hdg.get(), [](const void *c, const Vec &a, Vec &b) { static_cast<const HybridOperator *>(c)->apply(a, b); }},
                          Action{h->pc_hdg.get(), [](const void *c, const Vec &a, Vec &b) { static_cast<const BlockJacobi *>(c)->apply(a, b); }},
                          vec(rhs, n), xv, limit, tol);
        out(xv, x);
        out(g.residual(), residual);
        *iters = res.iterations;
        *rel = res.relative_residual;
    });
}
// Runs the integrator; stats8 = final_time, drift, newton, krylov, steps, max_lin, max_dg, seconds.
// updates (optional) receives up to max_updates rows of 13 doubles:
// step, stage, iteration, krylov, time, stage_time, dt, cfl, rms, damping, lin_rel, dg_rel, seconds
int oracle_advance(void *hv, int method, double *u, double *stats8, double *updates, int max_updates,
                   int *n_updates) {
    auto *h = static_cast<Handle *>(hv);
    return guard([&] {
        Vec s = vec(u, h->p->size());
        RunStatistics st = advance(*h->p, method == 0 ? Method::DG : Method::HDG, s);
        out(s, u);
        stats8[0] = st.final_time; stats8[1] = st.conservation_drift; stats8[2] = st.newton_iterations;
        stats8[3] = st.krylov_iterations; stats8[4] = st.steps; stats8[5] = st.max_linear_residual;
        stats8[6] = st.max_dg_linear_residual; stats8[7] = st.seconds;
        int k = 0;
        for (; k < (int)st.updates.size() && k < max_updates && updates; ++k) {
            const auto &x = st.updates[k];
            double row[13] = {(double)x.step, (double)x.stage, (double)x.iteration, (double)x.krylov_iterations,
                              x.time, x.stage_time, x.dt, x.cfl, x.residual_physical_rms, x.damping,
                              x.linear_relative_residual, x.dg_linear_relative_residual, x.iteration_s};
            std::memcpy(updates + 13 * k, row, sizeof(row));
        }
        *n_updates = (int)st.updates.size();
    });
}
// The exactness property the reference's own check asserts for block ILU(0)
// (dg_hdg_1d/check/check_1d.cpp:109-138): on a block path graph (natural ordering) and on a
// full block graph ILU(0) has no dropped fill, so one application solves A x = A exact.
// Off-diagonal blocks 0.03 * uniform[-1, 1) from a fixed LCG, diagonal blocks the cyclic
// shift with entries 3 + v.  Returns max |x - exact| in *err.
int oracle_ilu_exactness(int count, int width, int full, double *err) {
    return guard([&] {
        std::vector<std::vector<int>> adj(count);
        for (int i = 0; i < count; ++i)
            for (int j = 0; j < count; ++j)
                if (full || std::abs(i - j) <= 1) adj[i].push_back(j);
        unsigned long long state = 12345;
        auto uniform = [&] {
            state = state * 6364136223846793005ULL + 1442695040888963407ULL;
            return (double)(state >> 11) / 9007199254740992.0 * 2 - 1;
        };
        const size_t w2 = (size_t)width * width;
        std::map<std::pair<int, int>, Vec> blocks;
        for (int i = 0; i < count; ++i)
            for (int j : adj[i]) {
                Vec b(w2, 0.);
                if (i == j) {
                    for (int v = 0; v < width; ++v) b[(size_t)((v + 1) % width) * width + v] = 3 + v;
                } else {
                    for (auto &x : b) x = .03 * uniform();
                }
                blocks[{i, j}] = b;
            }
        Vec exact((size_t)count * width), rhs((size_t)count * width, 0.), x;
        for (size_t i = 0; i < exact.size(); ++i) exact[i] = std::sin(1.0 + 0.37 * (double)i);
        for (auto &[key, b] : blocks)
            for (int c = 0; c < width; ++c)
                for (int r = 0; r < width; ++r)
                    rhs[(size_t)key.first * width + r] += b[(size_t)c * width + r] * exact[(size_t)key.second * width + c];
        oracle::BlockILU0 ilu(adj, width);
        ilu.refresh([&](int r, int c, double *o) {
            const Vec &b = blocks.at({r, c});
            std::copy(b.begin(), b.end(), o);
        });
        ilu.apply(rhs, x);
        double e = 0;
        for (size_t i = 0; i < x.size(); ++i) e = std::max(e, std::abs(x[i] - exact[i]));
        *err = e;
    });
}
}
