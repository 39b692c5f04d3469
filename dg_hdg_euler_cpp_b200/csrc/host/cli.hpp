// Table-driven command-line flags for the dgh2d / dgh1d front ends.  Each flag names how its
// value is read (an integer, a real, free text, one of a fixed set of words, or no value) and
// what it writes; the texts of the errors are the ones the reference's front ends print
// (dg_hdg_2d/src/config.cpp, dg_hdg_1d/src/config.cpp), which its drivers and tests match.
#pragma once

#include <algorithm>
#include <cstdlib>
#include <functional>
#include <initializer_list>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

namespace dghcli {

inline void require(bool ok, const std::string &message) {
    if (!ok) throw std::runtime_error(message);
}

inline int to_int(const std::string &text) {
    std::size_t used = 0;
    int v = 0;
    try {
        v = std::stoi(text, &used);
    } catch (const std::exception &) {
        throw std::runtime_error("Invalid integer");
    }
    require(used == text.size(), "Invalid integer");
    return v;
}

inline double to_real(const std::string &text) {
    std::size_t used = 0;
    double v = 0;
    try {
        v = std::stod(text, &used);
    } catch (const std::exception &) {
        throw std::runtime_error("Invalid number");
    }
    require(used == text.size(), "Invalid number");
    return v;
}

// Returns the position of `text` in `words`, or throws `message`.
inline int pick(const std::string &text, std::initializer_list<const char *> words, const std::string &message) {
    int i = 0;
    for (const char *w : words) {
        if (text == w) return i;
        ++i;
    }
    throw std::runtime_error(message);
}

struct Flag {
    std::string name;
    bool takes_value;
    std::function<void(const std::string &)> apply;  // receives the value ("" for a switch)
};

inline Flag integer(const std::string &name, std::function<void(int)> set) {
    return {name, true, [set](const std::string &t) { set(to_int(t)); }};
}
inline Flag real(const std::string &name, std::function<void(double)> set) {
    return {name, true, [set](const std::string &t) { set(to_real(t)); }};
}
inline Flag text(const std::string &name, std::function<void(const std::string &)> set) {
    return {name, true, std::move(set)};
}
inline Flag on(const std::string &name, std::function<void()> set) {
    return {name, false, [set](const std::string &) { set(); }};
}

// Applies argv[1..] against the table; `--help` prints `usage` and exits.
inline void apply_flags(int argc, char **argv, const std::vector<Flag> &table, const char *usage) {
    for (int i = 1; i < argc; ++i) {
        const std::string name = argv[i];
        if (name == "--help") {
            std::cout << usage;
            std::exit(0);
        }
        const Flag *hit = nullptr;
        for (const Flag &f : table)
            if (f.name == name) hit = &f;
        if (!hit) throw std::runtime_error("Unknown option: " + name);
        std::string value;
        if (hit->takes_value) {
            require(i + 1 < argc, "Missing option value");
            value = argv[++i];
        }
        hit->apply(value);
    }
}

}  // namespace dghcli

// ---- pieces both front ends write in the same form ----------------------------------------------
#include "dgh_gpu.h"

#include <cmath>
#include <fstream>
#include <iomanip>
#include <sys/stat.h>

namespace dghcli {

// Creates the directories of an output prefix ("a/b/run" -> a, a/b).
inline void make_parent_dirs(const std::string &prefix) {
    for (std::size_t at = prefix.find('/', 1); at != std::string::npos; at = prefix.find('/', at + 1))
        mkdir(prefix.substr(0, at).c_str(), 0755);
}

inline std::ofstream open_csv(const std::string &path, const char *header, const char *what) {
    std::ofstream out(path);
    require(bool(out), what);
    out << std::setprecision(17) << header;
    return out;
}

constexpr const char *kUpdateHeader =
    "method,step,stage,iteration,time,stage_time,dt,cfl,residual_physical_rms,damping,"
    "krylov_iterations,linear_relative_residual,dg_linear_relative_residual,iteration_s,measured\n";

// One CSV row per recorded Newton update (time_integrator.hpp:9-13); the first `warmup`
// updates are marked unmeasured.
inline void write_updates(std::ostream &out, const std::string &method, const std::vector<dgh_update_stats> &rows,
                          int recorded, int warmup) {
    const int shown = std::min<int>(recorded, (int)rows.size());
    for (int i = 0; i < shown; ++i) {
        const dgh_update_stats &u = rows[i];
        out << method << ',' << u.step << ',' << u.stage << ',' << u.iteration << ',' << u.time << ','
            << u.stage_time << ',' << u.dt << ',' << u.cfl << ',' << u.residual_physical_rms << ',' << u.damping
            << ',' << u.krylov_iterations << ',' << u.linear_relative_residual << ','
            << u.dg_linear_relative_residual << ',' << u.iteration_s << ',' << (i >= warmup) << '\n';
    }
}

inline double mean_newton_seconds(const dgh_run_stats &st) {
    return st.measured_updates ? st.measured_newton_seconds / st.measured_updates : 0.;
}

// The run statistics columns shared by both summaries, from `steps` to `mean_newton_s`.
inline void write_run_columns(std::ostream &out, const dgh_run_stats &st) {
    out << st.steps << ',' << st.final_time << ',' << st.newton_iterations << ',' << st.krylov_iterations << ','
        << st.max_linear_residual << ',' << st.max_dg_linear_residual << ',' << st.minimum_step << ','
        << st.maximum_step << ',' << (st.steps ? st.final_time / st.steps : 0.) << ',' << st.seconds << ','
        << st.measured_updates << ',' << mean_newton_seconds(st);
}

inline void print_run(const std::string &method, const dgh_run_stats &st) {
    std::cout << method << ": steps=" << st.steps << ", Newton=" << st.newton_iterations
              << ", Krylov=" << st.krylov_iterations << ", time=" << st.seconds
              << " s, mean Newton=" << mean_newton_seconds(st) << " s, conservation drift=" << st.conservation_drift
              << '\n';
}

// One context + integrator run of a method from the projected initial state; returns the final
// state and fills the statistics and update rows.  Owns and releases every device object.
struct MethodRun {
    std::vector<double> state;
    dgh_run_stats stats{};
    std::vector<dgh_update_stats> rows;
    double l2[4] = {0, 0, 0, 0};
    int64_t volume = 0, trace = 0;
    int n = 0, block = 0, cells = 0;
    double geometry[4] = {0, 0, 0, 0};
    std::vector<double> nodes, weights;
};

inline MethodRun run_method(dgh_config cfg, int method, bool graph, bool with_error) {
    cfg.method = method;
    MethodRun out;
    dgh_ctx *ctx = nullptr;
    if (dgh_ctx_create(&cfg, &ctx) != DGH_OK) throw std::runtime_error(dgh_last_error(nullptr));
    dgh_integrator *integ = nullptr;
    double *dev = nullptr;
    auto release = [&]() {
        if (integ) dgh_integrator_destroy(integ);
        if (dev) dgh_vec_free(ctx, dev);
        dgh_ctx_destroy(ctx);
    };
    try {
        auto check = [&](int rc) {
            if (rc != DGH_OK) throw std::runtime_error(dgh_last_error(ctx));
        };
        if (graph) check(dgh_gmres_graph_enable(ctx, 1));
        int64_t sz[8];
        check(dgh_sizes(ctx, sz));
        out.volume = sz[0];
        out.trace = sz[1];
        out.block = (int)sz[2];
        out.cells = (int)sz[3];
        out.n = (int)sz[5];
        check(dgh_geometry(ctx, out.geometry));
        out.nodes.resize(out.n);
        out.weights.resize(out.n);
        check(dgh_nodes(ctx, out.nodes.data(), out.weights.data()));
        check(dgh_vec_alloc(ctx, out.volume, &dev));
        check(dgh_initial(ctx, dev));
        out.state.resize(out.volume);
        check(dgh_download(ctx, out.state.data(), dev, out.volume));
        check(dgh_integrator_create(ctx, method, &integ));
        out.rows.resize(100000);
        if (dgh_advance(integ, out.state.data(), &out.stats, out.rows.data(), (int)out.rows.size()) != DGH_OK)
            throw std::runtime_error(dgh_integrator_error(integ));
        if (with_error) {
            check(dgh_upload(ctx, dev, out.state.data(), out.volume));
            check(dgh_l2_error(ctx, dev, out.stats.final_time, out.l2));
        } else {
            for (double &e : out.l2) e = std::nan("");
        }
    } catch (...) {
        release();
        throw;
    }
    release();
    return out;
}

}  // namespace dghcli
