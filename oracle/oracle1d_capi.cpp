// Test infrastructure only: C entry points of the 1D CPU oracle (dgh1d_oracle.hpp), loaded by
// tests/ through ctypes.  Each function mirrors one call of the reference's 1D solver surface
// (dg_hdg_1d/include/euler/*).  Functions return 0 on success and 1 on a thrown require();
// oracle_error() (oracle_capi.cpp) gives the text.
#include "dgh1d_oracle.hpp"

#include <cstring>
#include <memory>
#include <sstream>

using namespace oracle1d;

extern "C" void oracle_set_error(const char *m);  // oracle_capi.cpp

namespace {
struct Handle1 {
    std::unique_ptr<Problem> p;
    std::unique_ptr<DGOperator> dg;
    std::unique_ptr<HybridOperator> hdg;
    std::vector<oracle::DenseLU> pc_dg, pc_hdg;
    std::unique_ptr<oracle::BlockILU0> ilu_dg, ilu_hdg;  // --precond block-ilu0
};
template <class F> int guard(F &&f) {
    try {
        f();
        return 0;
    } catch (const std::exception &e) {
        oracle_set_error(e.what());
        return 1;
    }
}
Config config_from(const char *args) {
    std::istringstream in(args ? args : "");
    std::vector<std::string> words{"oracle1d"};
    for (std::string w; in >> w;) words.push_back(w);
    std::vector<char *> argv;
    for (auto &w : words) argv.push_back(w.data());
    return parse((int)argv.size(), argv.data());
}
Vec vec(const double *p, size_t n) { return Vec(p, p + n); }
void out(const Vec &v, double *p) { std::memcpy(p, v.data(), v.size() * sizeof(double)); }
Handle1 *H(void *h) { return static_cast<Handle1 *>(h); }
void factor(std::vector<oracle::DenseLU> &lus, int blocks, int width,
            const std::function<void(int, int, double *)> &provider) {
    lus.assign(blocks, oracle::DenseLU{});
    Vec blk((size_t)width * width);
    for (int i = 0; i < blocks; ++i) {
        provider(i, i, blk.data());
        lus[i].compute(blk.data(), width);
    }
}
void solve_all(const std::vector<oracle::DenseLU> &lus, int width, const Vec &x, Vec &z) {
    z.assign(x.size(), 0.);
    for (size_t i = 0; i < lus.size(); ++i) lus[i].solve(&x[i * width], &z[i * width]);
}
}  // namespace

extern "C" {
int oracle1d_run(int argc, char **argv) { return run_main(argc, argv); }
void *oracle1d_create(const char *args) {
    Handle1 *h = nullptr;
    if (guard([&] {
            auto c = config_from(args);
            h = new Handle1;
            h->p = std::make_unique<Problem>(c);
            h->dg = std::make_unique<DGOperator>(*h->p);
            h->hdg = std::make_unique<HybridOperator>(*h->p);
        }))
        return nullptr;
    return h;
}
void oracle1d_destroy(void *h) { delete H(h); }
// sizes: volume size, trace size, block width, cells, nodes, quadrature points
int oracle1d_sizes(void *h, long long *s) {
    s[0] = H(h)->p->size(); s[1] = (long long)H(h)->p->cells * NVAR; s[2] = H(h)->p->block;
    s[3] = H(h)->p->cells; s[4] = H(h)->p->n; s[5] = H(h)->p->basis.points;
    return 0;
}
int oracle1d_basis(void *h, double *x, double *w, double *values, double *wd) {
    const Basis &b = H(h)->p->basis;
    if (x) out(b.x, x);
    if (w) out(b.w, w);
    if (values) out(b.values, values);
    if (wd) out(b.wd, wd);
    return 0;
}
int oracle1d_mass(void *h, double *m) { out(H(h)->p->mass, m); return 0; }
int oracle1d_initial(void *h, double *u) {
    return guard([&] { Vec v; H(h)->p->initial(v); out(v, u); });
}
int oracle1d_exact(void *h, double x, double t, double *s) {
    return guard([&] { State e = H(h)->p->example.exact(x, t); for (int v = 0; v < NVAR; ++v) s[v] = e[v]; });
}
int oracle1d_freeze(void *h, const double *u, double *rate) {
    return guard([&] { *rate = H(h)->p->freeze(vec(u, H(h)->p->size())); });
}
int oracle1d_speeds(void *h, double *ab) {
    const auto &s = H(h)->p->speeds;
    for (size_t i = 0; i < s.size(); ++i) { ab[2 * i] = s[i].a; ab[2 * i + 1] = s[i].b; }
    return 0;
}
int oracle1d_set_stage(void *h, const double *old, double step) {
    H(h)->p->old = vec(old, H(h)->p->size());
    H(h)->p->step_size = step;
    return 0;
}
int oracle1d_residual(void *h, const double *u, double *r) {
    return guard([&] { Vec o; H(h)->p->dg_residual(vec(u, H(h)->p->size()), o); out(o, r); });
}
int oracle1d_trace(void *h, const double *u, double *lam) {
    return guard([&] { Vec o; H(h)->p->trace(vec(u, H(h)->p->size()), o); out(o, lam); });
}
int oracle1d_admissible(void *h, const double *u, int *ok) {
    return guard([&] { *ok = H(h)->p->admissible(vec(u, H(h)->p->size())) ? 1 : 0; });
}
int oracle1d_integral(void *h, const double *u, double *s) {
    State i = H(h)->p->integral(vec(u, H(h)->p->size()));
    for (int v = 0; v < NVAR; ++v) s[v] = i[v];
    return 0;
}
int oracle1d_l2_error(void *h, const double *u, double t, double *s) {
    return guard([&] { State e = H(h)->p->error(vec(u, H(h)->p->size()), t); for (int v = 0; v < NVAR; ++v) s[v] = e[v]; });
}
int oracle1d_dg_refresh(void *h, const double *u) {
    return guard([&] { H(h)->dg->refresh(vec(u, H(h)->p->size())); });
}
int oracle1d_dg_apply(void *h, const double *d, double *o) {
    return guard([&] { Vec r; H(h)->dg->apply(vec(d, H(h)->p->size()), r); out(r, o); });
}
int oracle1d_dg_block(void *h, int row, int col, double *o) {
    return guard([&] { H(h)->dg->block(row, col, o); });
}
int oracle1d_dg_precond_refresh(void *h) {
    return guard([&] {
        Handle1 *k = H(h);
        auto provider = [&](int r, int c, double *o) { k->dg->block(r, c, o); };
        if (k->p->config.ilu) {
            k->ilu_dg = std::make_unique<oracle::BlockILU0>(oracle::periodic_adjacency(k->p->cells), k->p->block);
            k->ilu_dg->refresh(provider);
        } else {
            factor(k->pc_dg, k->p->cells, k->p->block, provider);
        }
    });
}
int oracle1d_dg_precond_apply(void *h, const double *x, double *z) {
    return guard([&] {
        Vec o;
        if (H(h)->ilu_dg) H(h)->ilu_dg->apply(vec(x, H(h)->p->size()), o);
        else solve_all(H(h)->pc_dg, H(h)->p->block, vec(x, H(h)->p->size()), o);
        out(o, z);
    });
}
int oracle1d_hdg_refresh(void *h, const double *u, const double *r) {
    return guard([&] { H(h)->hdg->refresh_projected(vec(u, H(h)->p->size()), vec(r, H(h)->p->size())); });
}
int oracle1d_hdg_rhs(void *h, double *o) { out(H(h)->hdg->rhs(), o); return 0; }
int oracle1d_hdg_apply(void *h, const double *d, double *o) {
    return guard([&] { Vec r; H(h)->hdg->apply(vec(d, (size_t)H(h)->p->cells * NVAR), r); out(r, o); });
}
int oracle1d_hdg_block(void *h, int row, int col, double *o) {
    return guard([&] { H(h)->hdg->block(row, col, o); });
}
int oracle1d_hdg_recover(void *h, const double *d, double *o) {
    return guard([&] { Vec r; H(h)->hdg->recover(vec(d, (size_t)H(h)->p->cells * NVAR), r); out(r, o); });
}
// hybrid.cpp:118-130: the DG residual implied by the Schur error S dl - rhs.
int oracle1d_hdg_recovered_residual(void *h, const double *dl, double *o) {
    return guard([&] { Vec r; H(h)->hdg->recovered_residual(vec(dl, (size_t)H(h)->p->cells * NVAR), r); out(r, o); });
}
int oracle1d_hdg_precond_refresh(void *h) {
    return guard([&] {
        Handle1 *k = H(h);
        auto provider = [&](int r, int c, double *o) { k->hdg->block(r, c, o); };
        if (k->p->config.ilu) {
            k->ilu_hdg = std::make_unique<oracle::BlockILU0>(oracle::periodic_adjacency(k->p->cells), NVAR);
            k->ilu_hdg->refresh(provider);
        } else {
            factor(k->pc_hdg, k->p->cells, NVAR, provider);
        }
    });
}
int oracle1d_hdg_precond_apply(void *h, const double *x, double *z) {
    return guard([&] {
        Vec o;
        if (H(h)->ilu_hdg) H(h)->ilu_hdg->apply(vec(x, (size_t)H(h)->p->cells * NVAR), o);
        else solve_all(H(h)->pc_hdg, NVAR, vec(x, (size_t)H(h)->p->cells * NVAR), o);
        out(o, z);
    });
}
// op 0: DG J*v with block Jacobi, weights M^-1; op 1: Schur apply with face blocks, weights 1
// (dg_hdg_1d/src/time_integrator.cpp:27).
int oracle1d_gmres(void *h, int op, int restart, const double *rhs, double *x, int limit, double tol, int *iters,
                   double *rel, double *residual) {
    return guard([&] {
        Handle1 *k = H(h);
        const int n = op == 0 ? k->p->size() : k->p->cells * NVAR;
        oracle::GMRES g(n, restart, op == 0 ? k->p->inverse_mass : Vec(n, 1.));
        Vec xv;
        oracle::LinearResult res;
        struct Pc { const std::vector<oracle::DenseLU> *lus; int width; const oracle::BlockILU0 *ilu; };
        Pc pc{op == 0 ? &k->pc_dg : &k->pc_hdg, op == 0 ? k->p->block : NVAR,
              op == 0 ? k->ilu_dg.get() : k->ilu_hdg.get()};
        const oracle::Action M{&pc, [](const void *c, const Vec &a, Vec &b) {
                                   const Pc *q = static_cast<const Pc *>(c);
                                   if (q->ilu) q->ilu->apply(a, b);
                                   else solve_all(*q->lus, q->width, a, b);
                               }};
        if (op == 0)
            res = g.solve(oracle::Action{k->dg.get(), [](const void *c, const Vec &a, Vec &b) {
                              static_cast<const DGOperator *>(c)->apply(a, b);
                          }},
                          M, vec(rhs, n), xv, limit, tol);
        else
            res = g.solve(oracle::Action{k->hdg.get(), [](const void *c, const Vec &a, Vec &b) {
                              static_cast<const HybridOperator *>(c)->apply(a, b);
                          }},
                          M, vec(rhs, n), xv, limit, tol);
        out(xv, x);
        out(g.residual(), residual);
        *iters = res.iterations;
        *rel = res.relative_residual;
    });
}
// Same row format as oracle_advance (oracle_capi.cpp).
int oracle1d_advance(void *h, int method, double *u, double *stats8, double *updates, int max_updates,
                     int *n_updates) {
    return guard([&] {
        Vec s = vec(u, H(h)->p->size());
        oracle::RunStatistics st = advance(*H(h)->p, method == 0 ? Method::DG : Method::HDG, s);
        out(s, u);
        stats8[0] = st.final_time; stats8[1] = st.conservation_drift; stats8[2] = st.newton_iterations;
        stats8[3] = st.krylov_iterations; stats8[4] = st.steps; stats8[5] = st.max_linear_residual;
        stats8[6] = st.max_dg_linear_residual; stats8[7] = st.seconds;
        for (int k = 0; k < (int)st.updates.size() && k < max_updates && updates; ++k) {
            const auto &x = st.updates[k];
            double row[13] = {(double)x.step, (double)x.stage, (double)x.iteration, (double)x.krylov_iterations,
                              x.time, x.stage_time, x.dt, x.cfl, x.residual_physical_rms, x.damping,
                              x.linear_relative_residual, x.dg_linear_relative_residual, x.iteration_s};
            std::memcpy(updates + 13 * k, row, sizeof(row));
        }
        *n_updates = (int)st.updates.size();
    });
}
}
