// dgh2d: command-line front end of the B200 solver, flag- and CSV-compatible with the
// reference's dg_hdg_2d (its flags and their error texts: dg_hdg_2d/src/config.cpp:23-122; its
// output files and columns: dg_hdg_2d/src/main.cpp:7-108).  Additional flags: --precision
// fp64|mixed|mixed16 (block-Jacobi factor precision), --condensation fp64|fp32, --graph, --autotune and
// --device N.
#include "cli.hpp"

namespace {
using dghcli::require;

struct Settings {
    dgh_config cfg{};
    std::string prefix = "output/run_2d";
    int methods = DGH_METHOD_BOTH;
    bool graph = false, timing_only = false, save_solution = true;
};

constexpr const char *kUsage =
    "2D periodic tensor-product Euler DG / condensed HDG on one B200\n"
    "--nx NX --ny NY --testcase diagonal|wave|axis --k K --quad Q --cfl C (--T T | --steps N)\n"
    "--method dg|hdg|both --linear gmres --precond block-jacobi|block-ilu0 (dg)\n"
    "--ordering natural --restart N --max-linear N --max-newton N\n"
    "--ntol R --ltol R --safety S --prefix PATH\n"
    "--integrator ssp-dirk3|be --newton-steps N --warmup-updates N\n"
    "--graph --autotune --timing-only --check-update --no-save-solution --precision fp64|mixed|mixed16\n"
    "--condensation fp64|fp32 --forcing 0|1 --device N\n";

Settings settings_from(int argc, char **argv) {
    Settings s;
    dgh_config &c = s.cfg;
    dgh_config_default(&c);
    int time_given = 0, steps_given = 0, direct = 0, method = -1, integrator = DGH_INTEGRATOR_DIRK3, testcase = 0;
    int ilu = 0, colamd = 0;
    std::string method_word = "both", integrator_word = "ssp-dirk3", testcase_word = "diagonal";
    using namespace dghcli;
    const std::vector<Flag> flags = {
        integer("--nx", [&](int v) { c.nx = v; }),
        integer("--ny", [&](int v) { c.ny = v; }),
        integer("--k", [&](int v) { c.degree = v; }),
        integer("--quad", [&](int v) { c.quadrature = v; }),
        real("--cfl", [&](double v) { c.cfl = v; }),
        real("--T", [&](double v) { c.final_time = v; time_given = 1; }),
        integer("--steps", [&](int v) { c.steps = v; steps_given = 1; }),
        real("--safety", [&](double v) { c.safety = v; }),
        real("--ntol", [&](double v) { c.nonlinear_tolerance = v; }),
        real("--ltol", [&](double v) { c.linear_tolerance = v; }),
        integer("--restart", [&](int v) { c.restart = v; }),
        integer("--max-linear", [&](int v) { c.max_linear = v; }),
        integer("--max-newton", [&](int v) { c.max_newton = v; }),
        integer("--newton-steps", [&](int v) { c.newton_steps = v; }),
        integer("--warmup-updates", [&](int v) { c.warmup_updates = v; }),
        integer("--device", [&](int v) { c.device = v; }),
        text("--testcase", [&](const std::string &v) { testcase_word = v; }),
        text("--method", [&](const std::string &v) { method_word = v; }),
        text("--integrator", [&](const std::string &v) { integrator_word = v; }),
        text("--prefix", [&](const std::string &v) { s.prefix = v; }),
        text("--precision", [&](const std::string &v) {
            const int level = pick(v, {"fp64", "mixed", "mixed16"}, "Invalid precision");
            c.precision = level == 2 ? DGH_PRECISION_MIXED16 : level == 1 ? DGH_PRECISION_MIXED : DGH_PRECISION_FP64;
        }),
        text("--condensation", [&](const std::string &v) {
            c.condense32 = pick(v, {"fp64", "fp32"}, "Invalid condensation precision");
        }),
        text("--forcing", [&](const std::string &v) { c.forcing = pick(v, {"0", "1"}, "Invalid forcing"); }),
        text("--linear", [&](const std::string &v) { direct = pick(v, {"gmres", "direct"}, "Invalid linear solver"); }),
        text("--ordering", [&](const std::string &v) { colamd = pick(v, {"natural", "colamd"}, "Invalid ordering"); }),
        text("--precond", [&](const std::string &v) {
            // block-ilu0 is this front end's extension (the reference's 2D front end has block Jacobi only)
            ilu = pick(v, {"block-jacobi", "block-ilu0"}, "2D currently supports block-jacobi only");
        }),
        on("--no-save-solution", [&] { s.save_solution = false; }),
        on("--timing-only", [&] { s.timing_only = true; }),
        on("--check-update", [&] { c.check_update = 1; }),
        on("--graph", [&] { s.graph = true; }),
        on("--autotune", [&] { c.autotune = 1; }),
    };
    apply_flags(argc, argv, flags, kUsage);
    require(!(time_given && steps_given), "Choose either --T or --steps");
    require(!steps_given || c.steps > 0, "steps must be positive");
    integrator = pick(integrator_word, {"ssp-dirk3", "be"}, "Invalid integrator") ? DGH_INTEGRATOR_BE
                                                                                   : DGH_INTEGRATOR_DIRK3;
    testcase = pick(testcase_word, {"diagonal", "wave", "axis"}, "Invalid testcase");
    method = pick(method_word, {"dg", "hdg", "both"}, "Method must be dg, hdg, or both");
    require(!direct, "The dense --linear direct reference is a CPU-only check; use gmres");
    require(!(ilu && colamd), "The device solver implements the natural block ordering only");
    require(!ilu || method == 0, "2D block ILU(0) is built for the DG operator only (method dg)");
    c.preconditioner = ilu;
    c.integrator = integrator;
    c.testcase = testcase == 0 ? DGH_TEST_DIAGONAL : testcase == 1 ? DGH_TEST_WAVE : DGH_TEST_AXIS;
    s.methods = method == 0 ? DGH_METHOD_DG : method == 1 ? DGH_METHOD_HDG : DGH_METHOD_BOTH;
    return s;
}

// The analytic solution of example.cpp:13-39 at (x, y, t), for the solution file's exact columns.
void exact_state(int testcase, double x, double y, double t, double out[4]) {
    const double gamma = 3., pi = std::acos(-1.);
    if (testcase == DGH_TEST_WAVE) {
        const double rho = 1 + .2 * std::sin(pi * (x - t)) * std::sin(pi * (y - .5 * t));
        out[0] = rho;
        out[1] = rho;
        out[2] = .5 * rho;
        out[3] = 1 / (gamma - 1) + .625 * rho;
        return;
    }
    const double c45 = std::cos(pi / 4), s45 = std::sin(pi / 4);
    const bool rotated = testcase == DGH_TEST_DIAGONAL;
    const double s = rotated ? c45 * x + s45 * y : x;  // coordinate along the wave
    // The characteristic foot xi of s: xi + t (a + b sin(pi xi)) = s, a = (3 - gamma)/2,
    // b = (gamma + 1)/4, bracketed and solved by safeguarded Newton.
    const double a = (3 - gamma) / 2, b = (gamma + 1) / 4;
    double lo = s - t * (a + b), hi = s - t * (a - b), xi = s - t * a;
    for (int k = 0; k < 80; ++k) {
        const double f = xi + t * (a + b * std::sin(pi * xi)) - s;
        if (std::abs(f) < 2e-15) break;
        (f > 0 ? hi : lo) = xi;
        const double next = xi - f / (1 + t * b * pi * std::cos(pi * xi));
        xi = (next > lo && next < hi) ? next : .5 * (lo + hi);
    }
    const double wave = std::sin(pi * xi), speed = .5 * (2 + wave), sound = (gamma - 1) * (2 - wave) / 4;
    const double rho = std::pow(sound * sound / gamma, 1 / (gamma - 1));
    out[0] = rho;
    out[1] = rho * speed * (rotated ? c45 : 1.);
    out[2] = rotated ? rho * speed * s45 : 0.;
    out[3] = std::pow(rho, gamma) / (gamma - 1) + .5 * rho * speed * speed;
}

// Node position of local node i (x fastest) of a cell, from the cell centre and Gauss nodes.
void node_xy(const dghcli::MethodRun &r, int nx, int cell, int i, double &x, double &y) {
    const double *g = r.geometry;  // hx, hy, lx, ly
    x = -.5 * g[2] + g[0] * (cell % nx + .5) + .5 * g[0] * r.nodes[i % r.n];
    y = -.5 * g[3] + g[1] * (cell / nx + .5) + .5 * g[1] * r.nodes[i / r.n];
}

void write_summary(std::ostream &out, const std::string &name, const Settings &s, const dghcli::MethodRun &r,
                   const char *integrator) {
    const dgh_config &c = s.cfg;
    out << name << ',' << c.nx << ',' << c.ny << ',' << c.degree << ',' << (c.quadrature ? c.quadrature : r.n) << ','
        << c.cfl << ',' << integrator << ",gmres,block-jacobi,natural," << c.nonlinear_tolerance << ','
        << c.linear_tolerance << ',' << c.safety << ',' << c.newton_steps << ',' << c.warmup_updates << ',';
    dghcli::write_run_columns(out, r.stats);
    out << ',' << r.volume << ',' << r.trace;
    for (double e : r.l2) out << ',' << e;
    out << ',' << r.stats.conservation_drift << ',' << r.geometry[2] << ',' << r.geometry[3] << ','
        << (name == "dg" ? "dense" : "face-dense") << '\n';
}

void write_solution(std::ostream &out, const std::string &name, const Settings &s, const dghcli::MethodRun &r) {
    const int plane = r.n * r.n;
    for (int cell = 0; cell < r.cells; ++cell)
        for (int i = 0; i < plane; ++i) {
            double x, y, ex[4];
            node_xy(r, s.cfg.nx, cell, i, x, y);
            exact_state(s.cfg.testcase, x, y, r.stats.final_time, ex);
            out << name << ',' << cell << ',' << i << ',' << x << ',' << y;
            for (int v = 0; v < 4; ++v) out << ',' << r.state[(size_t)cell * r.block + v * plane + i];
            for (double e : ex) out << ',' << e;
            out << '\n';
        }
}

// DG against HDG: per-variable mass-weighted L2 differences, their joint norm and the largest
// nodal difference; the two discretisations agree to round-off (main.cpp's 1e-8 guard).
void write_difference(const std::string &prefix, const dghcli::MethodRun &dg, const dghcli::MethodRun &hdg) {
    const int plane = dg.n * dg.n;
    const double area = .25 * dg.geometry[0] * dg.geometry[1];
    double largest = 0, sum_all = 0, per_var[4] = {0, 0, 0, 0};
    for (int cell = 0; cell < dg.cells; ++cell)
        for (int v = 0; v < 4; ++v)
            for (int i = 0; i < plane; ++i) {
                const size_t at = (size_t)cell * dg.block + v * plane + i;
                const double d = dg.state[at] - hdg.state[at];
                largest = std::max(largest, std::abs(d));
                per_var[v] += d * d * area * dg.weights[i % dg.n] * dg.weights[i / dg.n];
            }
    auto out = dghcli::open_csv(prefix + "_difference.csv", "rho_L2,momentum_x_L2,momentum_y_L2,energy_L2,joint_L2,max_nodal\n",
                                "Cannot open comparison output");
    for (double sq : per_var) {
        out << std::sqrt(sq) << ',';
        sum_all += sq;
    }
    out << std::sqrt(sum_all) << ',' << largest << '\n';
    std::cout << "DG/HDG max difference=" << largest << '\n';
    require(largest < 1e-8, "DG/HDG solutions disagree");
}
}  // namespace

int main(int argc, char **argv) {
    try {
        const Settings s = settings_from(argc, argv);
        dghcli::make_parent_dirs(s.prefix);
        auto summary = dghcli::open_csv(
            s.prefix + "_summary.csv",
            "method,nx,ny,k,quad,cfl,integrator,linear,preconditioner,ordering,ntol,ltol,safety,"
            "fixed_newton_steps,warmup_updates,steps,final_time,newton_iterations,krylov_iterations,"
            "max_linear_relative_residual,max_dg_linear_relative_residual,min_step,max_step,mean_dt,"
            "time_loop_s,measured_updates,mean_newton_s,volume_dofs,trace_dofs,"
            "rho_L2,momentum_x_L2,momentum_y_L2,energy_L2,max_conservation_drift,lx,ly,jacobi_local\n",
            "Cannot open output files");
        auto iterations = dghcli::open_csv(s.prefix + "_iterations.csv", dghcli::kUpdateHeader, "Cannot open output files");
        const bool solutions = !s.timing_only && s.save_solution;
        std::ofstream solution;
        if (solutions)
            solution = dghcli::open_csv(s.prefix + "_solution.csv",
                                        "method,cell,node,x,y,rho,momentum_x,momentum_y,energy,rho_exact,"
                                        "momentum_x_exact,momentum_y_exact,energy_exact\n",
                                        "Cannot open solution output");
        const char *integrator = s.cfg.integrator == DGH_INTEGRATOR_BE ? "be" : "ssp-dirk3";
        std::vector<dghcli::MethodRun> done;
        for (int method : {DGH_METHOD_DG, DGH_METHOD_HDG}) {
            if (s.methods != DGH_METHOD_BOTH && s.methods != method) continue;
            const std::string name = method == DGH_METHOD_DG ? "dg" : "hdg";
            done.push_back(dghcli::run_method(s.cfg, method, s.graph, !s.timing_only));
            const dghcli::MethodRun &r = done.back();
            write_summary(summary, name, s, r, integrator);
            dghcli::write_updates(iterations, name, r.rows, r.stats.updates_recorded, s.cfg.warmup_updates);
            if (solutions) write_solution(solution, name, s, r);
            dghcli::print_run(name, r.stats);
        }
        if (done.size() == 2) write_difference(s.prefix, done[0], done[1]);
    } catch (const std::exception &e) {
        std::cerr << "ERROR: " << e.what() << '\n';
        return 1;
    }
    return 0;
}
