// dgh2d: command-line front end of the B200 solver, flag- and CSV-compatible with the
// reference's dg_hdg_2d (dg_hdg_2d/src/main.cpp:7-108, config.cpp:23-122).  Additional flags:
// --precision fp64|mixed (block-Jacobi factor precision) and --device N.
#include "dgh_gpu.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <stdexcept>
#include <string>
#include <sys/stat.h>
#include <vector>

namespace {
void require(bool c, const std::string &m) {
    if (!c) throw std::runtime_error(m);
}
struct Options {
    dgh_config cfg;
    std::string method = "both", prefix = "output/run_2d", integrator = "ssp-dirk3", testcase = "diagonal";
    bool graph = false;
    bool timing_only = false, save_solution = true, direct = false;
};
Options parse(int argc, char **argv) {
    Options o;
    dgh_config_default(&o.cfg);
    bool time_seen = false, steps_seen = false;
    for (int i = 1; i < argc; ++i) {
        std::string option = argv[i];
        auto value = [&]() {
            require(i + 1 < argc, "Missing option value");
            return std::string(argv[++i]);
        };
        auto integer = [&]() {
            auto t = value();
            std::size_t end;
            int n = std::stoi(t, &end);
            require(end == t.size(), "Invalid integer");
            return n;
        };
        auto real = [&]() {
            auto t = value();
            std::size_t end;
            double n = std::stod(t, &end);
            require(end == t.size(), "Invalid number");
            return n;
        };
        dgh_config &c = o.cfg;
        if (option == "--nx") c.nx = integer();
        else if (option == "--ny") c.ny = integer();
        else if (option == "--testcase") o.testcase = value();
        else if (option == "--no-save-solution") o.save_solution = false;
        else if (option == "--newton-steps") c.newton_steps = integer();
        else if (option == "--warmup-updates") c.warmup_updates = integer();
        else if (option == "--integrator") o.integrator = value();
        else if (option == "--timing-only") o.timing_only = true;
        else if (option == "--check-update") c.check_update = 1;
        else if (option == "--k") c.degree = integer();
        else if (option == "--quad") c.quadrature = integer();
        else if (option == "--cfl") c.cfl = real();
        else if (option == "--T") { c.final_time = real(); time_seen = true; }
        else if (option == "--steps") { c.steps = integer(); steps_seen = true; }
        else if (option == "--safety") c.safety = real();
        else if (option == "--method") o.method = value();
        else if (option == "--prefix") o.prefix = value();
        else if (option == "--ntol") c.nonlinear_tolerance = real();
        else if (option == "--ltol") c.linear_tolerance = real();
        else if (option == "--restart") c.restart = integer();
        else if (option == "--max-linear") c.max_linear = integer();
        else if (option == "--max-newton") c.max_newton = integer();
        else if (option == "--device") c.device = integer();
        else if (option == "--graph") o.graph = true;
        else if (option == "--autotune") c.autotune = 1;
        else if (option == "--precision") {
            auto p = value();
            require(p == "fp64" || p == "mixed", "Invalid precision");
            c.precision = p == "mixed" ? DGH_PRECISION_MIXED : DGH_PRECISION_FP64;
        } else if (option == "--linear") {
            auto name = value();
            require(name == "direct" || name == "gmres", "Invalid linear solver");
            o.direct = name == "direct";
        } else if (option == "--ordering") {
            auto order = value();
            require(order == "natural" || order == "colamd", "Invalid ordering");
        } else if (option == "--precond") {
            auto name = value();
            require(name == "block-jacobi", "2D currently supports block-jacobi only");
        } else if (option == "--help") {
            std::cout << "2D periodic tensor-product Euler DG / condensed HDG on one B200\n"
                         "--nx NX --ny NY --testcase diagonal|wave|axis --k K --quad Q --cfl C (--T T | --steps N)\n"
                         "--method dg|hdg|both --linear gmres --precond block-jacobi\n"
                         "--ordering natural --restart N --max-linear N --max-newton N\n"
                         "--ntol R --ltol R --safety S --prefix PATH\n"
                         "--integrator ssp-dirk3|be --newton-steps N --warmup-updates N\n"
                         "--graph --autotune --timing-only --check-update --no-save-solution --precision fp64|mixed --device N\n";
            std::exit(0);
        } else
            throw std::runtime_error("Unknown option: " + option);
    }
    require(!(time_seen && steps_seen), "Choose either --T or --steps");
    require(!steps_seen || o.cfg.steps > 0, "steps must be positive");
    require(o.integrator == "be" || o.integrator == "ssp-dirk3", "Invalid integrator");
    require(o.testcase == "diagonal" || o.testcase == "wave" || o.testcase == "axis", "Invalid testcase");
    require(o.method == "dg" || o.method == "hdg" || o.method == "both", "Method must be dg, hdg, or both");
    require(!o.direct, "The dense --linear direct reference is a CPU-only check; use gmres");
    o.cfg.integrator = o.integrator == "be" ? DGH_INTEGRATOR_BE : DGH_INTEGRATOR_DIRK3;
    o.cfg.testcase = o.testcase == "diagonal" ? DGH_TEST_DIAGONAL : o.testcase == "wave" ? DGH_TEST_WAVE : DGH_TEST_AXIS;
    return o;
}
// example.cpp:13-39 evaluated on the host for the solution CSV's exact columns.
void exact(int testcase, double x, double y, double t, double u[4]) {
    const double g = 3., pi = std::acos(-1.);
    const double cs = std::cos(45. * pi / 180.), sn = std::sin(45. * pi / 180.);
    if (testcase == DGH_TEST_WAVE) {
        double rho = 1 + .2 * std::sin(pi * (x - t)) * std::sin(pi * (y - .5 * t));
        u[0] = rho; u[1] = rho; u[2] = .5 * rho; u[3] = 1 / (g - 1) + .625 * rho;
        return;
    }
    const bool diagonal = testcase == DGH_TEST_DIAGONAL;
    if (diagonal) x = cs * x + sn * y;
    const double a = (3 - g) / 2, b = (g + 1) / 4;
    double lo = x - t * (a + b), hi = x - t * (a - b), xi = x - t * a;
    for (int it = 0; it < 80; ++it) {
        double f = xi + t * (a + b * std::sin(pi * xi)) - x;
        if (std::abs(f) < 2e-15) break;
        if (f > 0) hi = xi; else lo = xi;
        double z = xi - f / (1 + t * b * pi * std::cos(pi * xi));
        xi = z > lo && z < hi ? z : .5 * (lo + hi);
    }
    const double jm = std::sin(pi * xi), velocity = .5 * (2 + jm), sound = (g - 1) * (2 - jm) / 4;
    const double rho = std::pow(sound * sound / g, 1 / (g - 1));
    u[0] = rho;
    u[1] = rho * velocity * (diagonal ? cs : 1.);
    u[2] = diagonal ? rho * velocity * sn : 0.;
    u[3] = std::pow(rho, g) / (g - 1) + .5 * rho * velocity * velocity;
}
void mkdirs(const std::string &prefix) {
    auto slash = prefix.find_last_of('/');
    if (slash == std::string::npos) return;
    std::string dir = prefix.substr(0, slash), acc;
    for (size_t i = 0; i <= dir.size(); ++i) {
        if ((i == dir.size() || dir[i] == '/') && !acc.empty()) mkdir(acc.c_str(), 0755);
        if (i < dir.size()) acc += dir[i];
    }
}
}  // namespace

int main(int argc, char **argv) {
    try {
        const Options o = parse(argc, argv);
        const dgh_config &base = o.cfg;
        mkdirs(o.prefix);
        std::ofstream summary(o.prefix + "_summary.csv"), updates(o.prefix + "_iterations.csv");
        require(bool(summary) && bool(updates), "Cannot open output files");
        summary << std::setprecision(17)
                << "method,nx,ny,k,quad,cfl,integrator,linear,preconditioner,ordering,ntol,ltol,safety,"
                   "fixed_newton_steps,warmup_updates,steps,final_time,newton_iterations,krylov_iterations,"
                   "max_linear_relative_residual,max_dg_linear_relative_residual,min_step,max_step,mean_dt,"
                   "time_loop_s,measured_updates,mean_newton_s,volume_dofs,trace_dofs,"
                   "rho_L2,momentum_x_L2,momentum_y_L2,energy_L2,max_conservation_drift,lx,ly,jacobi_local\n";
        updates << std::setprecision(17)
                << "method,step,stage,iteration,time,stage_time,dt,cfl,residual_physical_rms,damping,"
                   "krylov_iterations,linear_relative_residual,dg_linear_relative_residual,iteration_s,measured\n";
        std::ofstream solution_file;
        if (!o.timing_only && o.save_solution) {
            solution_file.open(o.prefix + "_solution.csv");
            require(bool(solution_file), "Cannot open solution output");
            solution_file << std::setprecision(17)
                          << "method,cell,node,x,y,rho,momentum_x,momentum_y,energy,rho_exact,momentum_x_exact,"
                             "momentum_y_exact,energy_exact\n";
        }
        std::vector<double> dg_solution;
        bool have_dg = false;
        for (int method : {DGH_METHOD_DG, DGH_METHOD_HDG}) {
            const std::string name = method == DGH_METHOD_DG ? "dg" : "hdg";
            if (o.method != "both" && o.method != name) continue;
            dgh_config cfg = base;
            cfg.method = method;
            dgh_ctx *ctx = nullptr;
            if (dgh_ctx_create(&cfg, &ctx) != DGH_OK) throw std::runtime_error(dgh_last_error(nullptr));
            auto ck = [&](int rc) {
                if (rc != DGH_OK) throw std::runtime_error(dgh_last_error(ctx));
            };
            if (o.graph) ck(dgh_gmres_graph_enable(ctx, 1));
            int64_t s[8];
            ck(dgh_sizes(ctx, s));
            const int64_t N = s[0], NT = s[1];
            const int n = (int)s[5], plane = n * n, m = (int)s[2], cells = (int)s[3];
            double geo[4];
            ck(dgh_geometry(ctx, geo));
            std::vector<double> xn(n);
            ck(dgh_nodes(ctx, xn.data(), nullptr));
            double *dev = nullptr;
            ck(dgh_vec_alloc(ctx, N, &dev));
            ck(dgh_initial(ctx, dev));
            std::vector<double> solution(N);
            ck(dgh_download(ctx, solution.data(), dev, N));
            dgh_integrator *it = nullptr;
            ck(dgh_integrator_create(ctx, method, &it));
            std::vector<dgh_update_stats> rows(100000);
            dgh_run_stats st{};
            if (dgh_advance(it, solution.data(), &st, rows.data(), (int)rows.size()) != DGH_OK)
                throw std::runtime_error(dgh_integrator_error(it));
            double err[4];
            if (o.timing_only) {
                for (double &e : err) e = std::numeric_limits<double>::quiet_NaN();
            } else {
                ck(dgh_upload(ctx, dev, solution.data(), N));
                ck(dgh_l2_error(ctx, dev, st.final_time, err));
            }
            summary << name << ',' << base.nx << ',' << base.ny << ',' << base.degree << ','
                    << (base.quadrature ? base.quadrature : n) << ',' << base.cfl
                    << ',' << o.integrator << ",gmres,block-jacobi,natural," << base.nonlinear_tolerance << ','
                    << base.linear_tolerance << ',' << base.safety << ',' << base.newton_steps << ','
                    << base.warmup_updates << ',' << st.steps << ',' << st.final_time << ',' << st.newton_iterations
                    << ',' << st.krylov_iterations << ',' << st.max_linear_residual << ',' << st.max_dg_linear_residual
                    << ',' << st.minimum_step << ',' << st.maximum_step << ','
                    << (st.steps ? st.final_time / st.steps : 0.) << ',' << st.seconds << ',' << st.measured_updates
                    << ',' << (st.measured_updates ? st.measured_newton_seconds / st.measured_updates : 0.) << ','
                    << N << ',' << NT;
            for (double e : err) summary << ',' << e;
            summary << ',' << st.conservation_drift << ',' << geo[2] << ',' << geo[3] << ','
                    << (method == DGH_METHOD_DG ? "dense" : "face-dense") << '\n';
            const int nrec = std::min<int>(st.updates_recorded, (int)rows.size());
            for (int i = 0; i < nrec; ++i) {
                const auto &u = rows[i];
                updates << name << ',' << u.step << ',' << u.stage << ',' << u.iteration << ',' << u.time << ','
                        << u.stage_time << ',' << u.dt << ',' << u.cfl << ',' << u.residual_physical_rms << ','
                        << u.damping << ',' << u.krylov_iterations << ',' << u.linear_relative_residual << ','
                        << u.dg_linear_relative_residual << ',' << u.iteration_s << ','
                        << (i >= base.warmup_updates) << '\n';
            }
            if (!o.timing_only && o.save_solution)
                for (int cell = 0; cell < cells; ++cell)
                    for (int i = 0; i < plane; ++i) {
                        const double x = -.5 * geo[2] + geo[0] * (cell % base.nx + .5) + .5 * geo[0] * xn[i % n];
                        const double y = -.5 * geo[3] + geo[1] * (cell / base.nx + .5) + .5 * geo[1] * xn[i / n];
                        double ex[4];
                        exact(cfg.testcase, x, y, st.final_time, ex);
                        solution_file << name << ',' << cell << ',' << i << ',' << x << ',' << y;
                        for (int v = 0; v < 4; ++v) solution_file << ',' << solution[(size_t)cell * m + v * plane + i];
                        for (int v = 0; v < 4; ++v) solution_file << ',' << ex[v];
                        solution_file << '\n';
                    }
            std::cout << name << ": steps=" << st.steps << ", Newton=" << st.newton_iterations
                      << ", Krylov=" << st.krylov_iterations << ", time=" << st.seconds << " s, mean Newton="
                      << (st.measured_updates ? st.measured_newton_seconds / st.measured_updates : 0.)
                      << " s, conservation drift=" << st.conservation_drift << '\n';
            std::vector<double> mass(N);
            if (method == DGH_METHOD_DG && o.method == "both") {
                dg_solution = solution;
                have_dg = true;
            } else if (have_dg) {
                double maximum = 0;
                for (int64_t i = 0; i < N; ++i) maximum = std::max(maximum, std::abs(dg_solution[i] - solution[i]));
                std::ofstream comparison(o.prefix + "_difference.csv");
                require(bool(comparison), "Cannot open comparison output");
                std::vector<double> w(n);
                ck(dgh_nodes(ctx, nullptr, w.data()));
                comparison << std::setprecision(17) << "rho_L2,momentum_x_L2,momentum_y_L2,energy_L2,joint_L2,max_nodal\n";
                double joint = 0.;
                for (int v = 0; v < 4; ++v) {
                    double sq = 0.;
                    for (int cell = 0; cell < cells; ++cell)
                        for (int node = 0; node < plane; ++node) {
                            const size_t k = (size_t)cell * m + v * plane + node;
                            const double d = dg_solution[k] - solution[k];
                            sq += d * d * (.25 * geo[0] * geo[1] * w[node % n] * w[node / n]);
                        }
                    comparison << std::sqrt(sq) << ',';
                    joint += sq;
                }
                comparison << std::sqrt(joint) << ',' << maximum << '\n';
                std::cout << "DG/HDG max difference=" << maximum << '\n';
                require(maximum < 1e-8, "DG/HDG solutions disagree");
            }
            dgh_integrator_destroy(it);
            dgh_vec_free(ctx, dev);
            dgh_ctx_destroy(ctx);
        }
    } catch (const std::exception &e) {
        std::cerr << "ERROR: " << e.what() << '\n';
        return 1;
    }
    return 0;
}
