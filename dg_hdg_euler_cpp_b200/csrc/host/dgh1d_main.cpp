// dgh1d: command-line front end of the B200 solver for the 1D problem, flag- and CSV-compatible
// with the reference's dg_hdg_1d (its flags and their error texts: dg_hdg_1d/src/config.cpp:22-115;
// its output files and columns: dg_hdg_1d/src/main.cpp:7-107).  The device path implements GMRES
// with block Jacobi or block ILU(0) in the natural ordering; --ordering colamd with block-ilu0 and
// --linear direct are refused with a message.  Additional flags: --precision fp64|mixed (block
// factor precision), --graph and --device N.
#include "cli.hpp"

namespace {
using dghcli::require;

struct Settings {
    dgh_config cfg{};
    std::string prefix = "output/run";
    int methods = DGH_METHOD_BOTH;
    bool graph = false, timing_only = false;
};

constexpr const char *kUsage =
    "1D periodic Euler DG / condensed HDG on one B200\n"
    "--cells N --k K --quad Q --cfl C (--T T | --steps N)\n"
    "--method dg|hdg|both --linear gmres --precond block-jacobi|block-ilu0\n"
    "--ordering natural --restart N --max-linear N --max-newton N\n"
    "--ntol R --ltol R --safety S --prefix PATH\n"
    "--integrator ssp-dirk3|be --newton-steps N --warmup-updates N\n"
    "--graph --timing-only --check-update --precision fp64|mixed --device N\n";

Settings settings_from(int argc, char **argv) {
    Settings s;
    dgh_config &c = s.cfg;
    dgh_config_default(&c);
    c.dim = 1;
    c.nx = 32;  // dg_hdg_1d/include/euler/config.hpp:8
    c.ny = 1;
    int time_given = 0, steps_given = 0, direct = 0, ilu = 0, colamd = 0;
    std::string method_word = "both", integrator_word = "ssp-dirk3";
    using namespace dghcli;
    const std::vector<Flag> flags = {
        integer("--cells", [&](int v) { c.nx = v; }),
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
        text("--method", [&](const std::string &v) { method_word = v; }),
        text("--integrator", [&](const std::string &v) { integrator_word = v; }),
        text("--prefix", [&](const std::string &v) { s.prefix = v; }),
        text("--precision", [&](const std::string &v) {
            c.precision = pick(v, {"fp64", "mixed"}, "Invalid precision") ? DGH_PRECISION_MIXED : DGH_PRECISION_FP64;
        }),
        text("--linear", [&](const std::string &v) { direct = pick(v, {"gmres", "direct"}, "Invalid linear solver"); }),
        text("--ordering", [&](const std::string &v) { colamd = pick(v, {"natural", "colamd"}, "Invalid ordering"); }),
        text("--precond", [&](const std::string &v) {
            ilu = pick(v, {"block-jacobi", "block-ilu0"}, "Invalid block preconditioner");
        }),
        on("--timing-only", [&] { s.timing_only = true; }),
        on("--check-update", [&] { c.check_update = 1; }),
        on("--graph", [&] { s.graph = true; }),
    };
    apply_flags(argc, argv, flags, kUsage);
    require(!(time_given && steps_given), "Choose either --T or --steps");
    require(!steps_given || c.steps > 0, "steps must be positive");
    c.integrator = pick(integrator_word, {"ssp-dirk3", "be"}, "Invalid integrator") ? DGH_INTEGRATOR_BE
                                                                                    : DGH_INTEGRATOR_DIRK3;
    const int method = pick(method_word, {"dg", "hdg", "both"}, "Method must be dg, hdg, or both");
    require(!direct, "The dense --linear direct reference is a CPU-only check; use gmres");
    require(!(ilu && colamd), "The device solver implements the natural block ordering only");
    c.preconditioner = ilu;
    s.methods = method == 0 ? DGH_METHOD_DG : method == 1 ? DGH_METHOD_HDG : DGH_METHOD_BOTH;
    return s;
}

// The analytic simple wave of dg_hdg_1d/src/simple_wave.cpp:3-25 at (x, t).
void exact_state(double x, double t, double out[3]) {
    const double gamma = 3., pi = std::acos(-1.), a = (3 - gamma) / 2, b = (gamma + 1) / 4;
    double lo = x - t * (a + b), hi = x - t * (a - b), xi = x - t * a;
    for (int k = 0; k < 80; ++k) {
        const double f = xi + t * (a + b * std::sin(pi * xi)) - x;
        if (std::abs(f) < 2e-15) break;
        (f > 0 ? hi : lo) = xi;
        const double next = xi - f / (1 + t * b * pi * std::cos(pi * xi));
        xi = (next > lo && next < hi) ? next : .5 * (lo + hi);
    }
    const double wave = std::sin(pi * xi), speed = .5 * (2 + wave), sound = (gamma - 1) * (2 - wave) / 4;
    const double rho = std::pow(sound * sound / gamma, 1 / (gamma - 1));
    out[0] = rho;
    out[1] = rho * speed;
    out[2] = std::pow(rho, gamma) / (gamma - 1) + .5 * rho * speed * speed;
}

void write_summary(std::ostream &out, const std::string &name, const Settings &s, const dghcli::MethodRun &r,
                   const char *integrator) {
    const dgh_config &c = s.cfg;
    out << name << ',' << r.cells << ',' << c.degree << ',' << (c.quadrature ? c.quadrature : r.n) << ',' << c.cfl
        << ',' << integrator << ",gmres," << (c.preconditioner ? "block-ilu0" : "block-jacobi") << ",natural,"
        << c.nonlinear_tolerance << ',' << c.linear_tolerance << ',' << c.safety << ',' << c.newton_steps << ','
        << c.warmup_updates << ',';
    dghcli::write_run_columns(out, r.stats);
    out << ',' << r.volume << ',' << r.trace;
    for (int v = 0; v < 3; ++v) out << ',' << r.l2[v];
    out << ',' << r.stats.conservation_drift << '\n';
}

void write_solution(std::ostream &out, const std::string &name, const dghcli::MethodRun &r) {
    const double h = r.geometry[0];
    for (int cell = 0; cell < r.cells; ++cell)
        for (int i = 0; i < r.n; ++i) {
            const double x = -1 + h * (cell + .5) + .5 * h * r.nodes[i];
            double ex[3];
            exact_state(x, r.stats.final_time, ex);
            out << name << ',' << cell << ',' << i << ',' << x;
            for (int v = 0; v < 3; ++v) out << ',' << r.state[(size_t)cell * r.block + v * r.n + i];
            for (double e : ex) out << ',' << e;
            out << '\n';
        }
}

void write_difference(const std::string &prefix, const dghcli::MethodRun &dg, const dghcli::MethodRun &hdg) {
    const double half_h = .5 * dg.geometry[0];
    double largest = 0, sum_all = 0, per_var[3] = {0, 0, 0};
    for (int cell = 0; cell < dg.cells; ++cell)
        for (int v = 0; v < 3; ++v)
            for (int i = 0; i < dg.n; ++i) {
                const size_t at = (size_t)cell * dg.block + v * dg.n + i;
                const double d = dg.state[at] - hdg.state[at];
                largest = std::max(largest, std::abs(d));
                per_var[v] += d * d * half_h * dg.weights[i];
            }
    auto out = dghcli::open_csv(prefix + "_difference.csv", "rho_L2,momentum_L2,energy_L2,joint_L2,max_nodal\n",
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
            "method,cells,k,quad,cfl,integrator,linear,preconditioner,ordering,ntol,ltol,safety,"
            "fixed_newton_steps,warmup_updates,steps,final_time,newton_iterations,krylov_iterations,"
            "max_linear_relative_residual,max_dg_linear_relative_residual,min_step,max_step,mean_dt,"
            "time_loop_s,measured_updates,mean_newton_s,volume_dofs,trace_dofs,"
            "rho_L2,momentum_L2,energy_L2,max_conservation_drift\n",
            "Cannot open output files");
        auto iterations = dghcli::open_csv(s.prefix + "_iterations.csv", dghcli::kUpdateHeader, "Cannot open output files");
        std::ofstream solution;
        if (!s.timing_only)
            solution = dghcli::open_csv(s.prefix + "_solution.csv",
                                        "method,cell,node,x,rho,momentum,energy,rho_exact,momentum_exact,energy_exact\n",
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
            if (!s.timing_only) write_solution(solution, name, r);
            dghcli::print_run(name, r.stats);
        }
        if (done.size() == 2) write_difference(s.prefix, done[0], done[1]);
    } catch (const std::exception &e) {
        std::cerr << "ERROR: " << e.what() << '\n';
        return 1;
    }
    return 0;
}
