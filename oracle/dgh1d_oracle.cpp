// Test infrastructure only: CPU restatement of the reference's 1D solver (dg_hdg_1d/), see
// dgh1d_oracle.hpp.  Every routine cites the reference file:line it follows.
#include "dgh1d_oracle.hpp"

#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>

namespace oracle1d {

// ---------------------------------------------------------------- dg_hdg_1d/src/config.cpp:6-21
void validate(const Config &c) {
    require(c.cells >= 3 && c.degree >= 0 && c.degree <= 8 && c.quadrature >= 0, "Invalid mesh or degree");
    require(c.quadrature == 0 || c.quadrature >= c.degree + 1, "Quadrature must be >= degree+1");
    require(c.restart > 0 && c.max_linear > 0 && c.max_newton > 0 && c.steps >= 0, "Invalid iteration limit");
    require(c.newton_steps >= 0 && c.warmup_updates >= 0, "Invalid timing update count");
    require(c.integrator == "be" || c.integrator == "ssp-dirk3", "Invalid integrator");
    require(std::isfinite(c.cfl) && c.cfl > 0 && std::isfinite(c.final_time) && c.final_time >= 0,
            "CFL must be positive and final time nonnegative");
    require(std::isfinite(c.safety) && c.safety >= 1 && std::isfinite(c.nonlinear_tolerance) &&
                c.nonlinear_tolerance > 0 && std::isfinite(c.linear_tolerance) && c.linear_tolerance > 0 &&
                c.linear_tolerance < 1,
            "Invalid solver tolerance or wave-speed safety");
    require(c.method == "dg" || c.method == "hdg" || c.method == "both", "Method must be dg, hdg, or both");
}

// ---------------------------------------------------------------- dg_hdg_1d/src/config.cpp:22-115
Config parse(int argc, char **argv) {
    Config c;
    bool time_seen = false, steps_seen = false;
    for (int i = 1; i < argc; ++i) {
        const std::string option = argv[i];
        auto value = [&]() {
            require(i + 1 < argc, "Missing option value");
            return std::string(argv[++i]);
        };
        auto integer = [&]() {
            const std::string text = value();
            size_t end = 0;
            const int v = std::stoi(text, &end);
            require(end == text.size(), "Invalid integer");
            return v;
        };
        auto real = [&]() {
            const std::string text = value();
            size_t end = 0;
            const double v = std::stod(text, &end);
            require(end == text.size(), "Invalid number");
            return v;
        };
        if (option == "--cells") c.cells = integer();
        else if (option == "--newton-steps") c.newton_steps = integer();
        else if (option == "--warmup-updates") c.warmup_updates = integer();
        else if (option == "--integrator") c.integrator = value();
        else if (option == "--timing-only") c.timing_only = true;
        else if (option == "--check-update") c.check_update = true;
        else if (option == "--k") c.degree = integer();
        else if (option == "--quad") c.quadrature = integer();
        else if (option == "--cfl") c.cfl = real();
        else if (option == "--T") {
            c.final_time = real();
            time_seen = true;
        } else if (option == "--steps") {
            c.steps = integer();
            steps_seen = true;
        } else if (option == "--safety") c.safety = real();
        else if (option == "--method") c.method = value();
        else if (option == "--prefix") c.prefix = value();
        else if (option == "--ntol") c.nonlinear_tolerance = real();
        else if (option == "--ltol") c.linear_tolerance = real();
        else if (option == "--restart") c.restart = integer();
        else if (option == "--max-linear") c.max_linear = integer();
        else if (option == "--max-newton") c.max_newton = integer();
        else if (option == "--linear") {
            const std::string name = value();
            require(name == "direct" || name == "gmres", "Invalid linear solver");
            c.direct = name == "direct";
        } else if (option == "--ordering") {
            const std::string order = value();
            require(order == "natural" || order == "colamd", "Invalid ordering");
            c.colamd = order == "colamd";
        } else if (option == "--precond") {
            const std::string name = value();
            require(name == "block-jacobi" || name == "block-ilu0", "Invalid block preconditioner");
            c.ilu = name == "block-ilu0";
        } else throw std::runtime_error("Unknown option: " + option);
    }
    require(!(time_seen && steps_seen), "Choose either --T or --steps");
    require(!steps_seen || c.steps > 0, "steps must be positive");
    validate(c);
    return c;
}

// ---------------------------------------------------------------- nodal_basis.hpp:12-66
Vec Basis::evaluate(double z) const {
    Vec v(nodes, 1.);
    for (int i = 0; i < nodes; ++i)
        for (int j = 0; j < nodes; ++j)
            if (i != j) v[i] *= (z - x[j]) / (x[i] - x[j]);
    return v;
}
Basis::Basis(int degree, int quadrature) : nodes(degree + 1), points(quadrature ? quadrature : degree + 1) {
    require(nodes > 0 && points >= nodes, "Require quadrature >= degree+1");
    const int n = nodes, Q = points;
    oracle::gauss(n, x, w);
    oracle::gauss(Q, qx, qw);
    Vec bary(n, 1.);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            if (i != j) bary[i] /= x[i] - x[j];
    Vec D(n * n, 0.);  // D[i*n+j] = l_j'(x_i)
    for (int i = 0; i < n; ++i) {
        double sum = 0;
        for (int j = 0; j < n; ++j)
            if (i != j) {
                D[i * n + j] = bary[j] / (bary[i] * (x[i] - x[j]));
                sum += D[i * n + j];
            }
        D[i * n + i] = -sum;
    }
    values.assign(Q * n, 0.);
    for (int q = 0; q < Q; ++q) {
        if (Q == n) {
            values[q * n + q] = 1.;  // nodal_basis.hpp:52-53: collocation uses the identity
            continue;
        }
        const Vec v = evaluate(qx[q]);
        for (int i = 0; i < n; ++i) values[q * n + i] = v[i];
    }
    wd.assign(Q * n, 0.);
    for (int q = 0; q < Q; ++q)
        for (int i = 0; i < n; ++i) {
            double s = 0;
            for (int j = 0; j < n; ++j) s += values[q * n + j] * D[j * n + i];
            wd[q * n + i] = qw[q] * s;
        }
    left = evaluate(-1);
    right = evaluate(1);
    oracle::gauss(std::max(20, 2 * n + 3), ex, ew);
    const int Qe = (int)ex.size();
    evalues.assign(Qe * n, 0.);
    for (int q = 0; q < Qe; ++q) {
        const Vec v = evaluate(ex[q]);
        for (int i = 0; i < n; ++i) evalues[q * n + i] = v[i];
    }
    projection.assign(n * Qe, 0.);
    for (int i = 0; i < n; ++i)
        for (int q = 0; q < Qe; ++q) projection[i * Qe + q] = evalues[q * n + i] * ew[q] / w[i];
}

// ---------------------------------------------------------------- dg_hdg_1d/src/physics.cpp:4-38
double Gas::pressure(const State &u) const {
    return (gamma - 1) * (u[Energy] - .5 * u[Momentum] * u[Momentum] / u[Density]);
}
State Gas::flux(const State &u) const {
    const double velocity = u[Momentum] / u[Density], p = pressure(u);
    return {u[Momentum], u[Momentum] * velocity + p, (u[Energy] + p) * velocity};
}
Jac Gas::jacobian(const State &u) const {
    const double v = u[Momentum] / u[Density], H = (u[Energy] + pressure(u)) / u[Density], g = gamma;
    return {0., 1., 0., .5 * (g - 3) * v * v, (3 - g) * v, g - 1, v * (.5 * (g - 1) * v * v - H),
            H - (g - 1) * v * v, g * v};
}
double Gas::spectral_radius(const State &u) const {
    return std::abs(u[Momentum] / u[Density]) + std::sqrt(gamma * pressure(u) / u[Density]);
}
Speed einfeldt(const State &l, const State &r, const Gas &gas, double safety) {
    require(l[Density] > 0 && r[Density] > 0 && gas.pressure(l) > 0 && gas.pressure(r) > 0,
            "Invalid frozen face state");
    const double sl = std::sqrt(l[Density]), sr = std::sqrt(r[Density]);
    const double ul = l[Momentum] / l[Density], ur = r[Momentum] / r[Density];
    const double cl = std::sqrt(gas.gamma * gas.pressure(l) / l[Density]);
    const double cr = std::sqrt(gas.gamma * gas.pressure(r) / r[Density]);
    const double v = (sl * ul + sr * ur) / (sl + sr);
    const double H = (sl * (l[Energy] + gas.pressure(l)) / l[Density] + sr * (r[Energy] + gas.pressure(r)) / r[Density]) /
                     (sl + sr);
    const double c = std::sqrt((gas.gamma - 1) * (H - .5 * v * v));
    return {safety * std::max({0.0, -ul + cl, -v + c}), safety * std::max({0.0, ur + cr, v + c})};
}

// ---------------------------------------------------------------- dg_hdg_1d/src/simple_wave.cpp:3-25
double SimpleWave::shock_time() const { return 4 / ((gas.gamma + 1) * std::acos(-1.0)); }
State SimpleWave::exact(double x, double t) const {
    require(t < shock_time(), "Simple wave reaches shock time");
    const double g = gas.gamma, pi = std::acos(-1.0), a = (3 - g) / 2, b = (g + 1) / 4;
    double lo = x - t * (a + b), hi = x - t * (a - b), xi = x - t * a;
    for (int i = 0; i < 80; ++i) {
        const double f = xi + t * (a + b * std::sin(pi * xi)) - x;
        if (std::abs(f) < 2e-15) break;
        if (f > 0) hi = xi;
        else lo = xi;
        const double z = xi - f / (1 + t * b * pi * std::cos(pi * xi));
        xi = z > lo && z < hi ? z : .5 * (lo + hi);
    }
    const double jm = std::sin(pi * xi), v = .5 * (2 + jm), c = (g - 1) * (2 - jm) / 4;
    const double rho = std::pow(c * c / g, 1 / (g - 1)), p = std::pow(rho, g);
    return {rho, rho * v, p / (g - 1) + .5 * rho * v * v};
}

// ---------------------------------------------------------------- dg_hdg_1d/src/discretization.cpp
Problem::Problem(const Config &c)
    : config(c), basis(c.degree, c.quadrature), cells(c.cells), n(basis.nodes), block(NVAR * basis.nodes),
      h(2.0 / c.cells) {
    validate(c);
    old.assign(size(), 0.);
    mass.assign(size(), 0.);
    inverse_mass.assign(size(), 0.);
    for (int cell = 0; cell < cells; ++cell)
        for (int v = 0; v < NVAR; ++v)
            for (int i = 0; i < n; ++i) mass[index(cell, v, i)] = .5 * h * basis.w[i];
    for (int i = 0; i < size(); ++i) inverse_mass[i] = 1 / mass[i];
    speeds.assign(cells, Speed{0, 0});
}
State Problem::sample(const Vec &u, int cell, const Vec &shape) const {
    State s{0., 0., 0.};
    for (int v = 0; v < NVAR; ++v)
        for (int i = 0; i < n; ++i) s[v] += shape[i] * u[index(cell, v, i)];
    return s;
}
State Problem::quadrature_state(const Vec &u, int cell, int q) const {
    if (basis.points == n) return {u[index(cell, 0, q)], u[index(cell, 1, q)], u[index(cell, 2, q)]};
    State s{0., 0., 0.};
    for (int v = 0; v < NVAR; ++v)
        for (int i = 0; i < n; ++i) s[v] += basis.values[q * n + i] * u[index(cell, v, i)];
    return s;
}
// discretization.cpp:31-74: L2 projection, then a convex limiter toward the cell mean so the
// state is admissible at the nodes, the quadrature points, the error points and both faces.
void Problem::initial(Vec &u) const {
    u.assign(size(), 0.);
    const int Qe = (int)basis.ex.size(), Q = basis.points;
    std::vector<State> samples(Qe), nodal(n), checks;
    for (int cell = 0; cell < cells; ++cell) {
        for (int q = 0; q < Qe; ++q) samples[q] = example.exact(-1 + h * (cell + .5) + .5 * h * basis.ex[q], 0);
        for (int i = 0; i < n; ++i) {
            State s{0., 0., 0.};
            for (int q = 0; q < Qe; ++q)
                for (int v = 0; v < NVAR; ++v) s[v] += basis.projection[i * Qe + q] * samples[q][v];
            nodal[i] = s;
        }
        State mean{0., 0., 0.};
        for (int v = 0; v < NVAR; ++v) {
            double s = 0;
            for (int i = 0; i < n; ++i) s += nodal[i][v] * basis.w[i];
            mean[v] = .5 * s;
        }
        require(mean[Density] > 0 && example.gas.pressure(mean) > 0, "Nonphysical cell average");
        checks.assign(nodal.begin(), nodal.end());
        auto combine = [&](const double *row) {
            State s{0., 0., 0.};
            for (int v = 0; v < NVAR; ++v)
                for (int i = 0; i < n; ++i) s[v] += row[i] * nodal[i][v];
            return s;
        };
        for (int q = 0; q < Q; ++q) checks.push_back(combine(&basis.values[q * n]));
        for (int q = 0; q < Qe; ++q) checks.push_back(combine(&basis.evalues[q * n]));
        checks.push_back(combine(basis.left.data()));
        checks.push_back(combine(basis.right.data()));
        double theta = 1;
        for (const State &z0 : checks) {
            State d;
            for (int v = 0; v < NVAR; ++v) d[v] = z0[v] - mean[v];
            auto physical = [&](double factor) {
                State z;
                for (int v = 0; v < NVAR; ++v) z[v] = mean[v] + factor * d[v];
                return z[Density] > 1e-12 && example.gas.pressure(z) > 1e-12;
            };
            if (!physical(theta)) {
                double low = 0, high = theta;
                for (int k = 0; k < 60; ++k) {
                    const double mid = .5 * (low + high);
                    if (physical(mid)) low = mid;
                    else high = mid;
                }
                theta = .99 * low;
            }
        }
        for (int v = 0; v < NVAR; ++v)
            for (int i = 0; i < n; ++i) u[index(cell, v, i)] = mean[v] + theta * (nodal[i][v] - mean[v]);
    }
    require(admissible(u), "Invalid projected initial state");
}
// discretization.cpp:75-92
double Problem::freeze(const Vec &u) {
    old = u;
    double rate = 0;
    for (int e = 0; e < cells; ++e)
        speeds[e] = einfeldt(sample(u, e, basis.right), sample(u, (e + 1) % cells, basis.left), example.gas,
                             config.safety);
    for (int e = 0; e < cells; ++e) {
        const Speed &l = speeds[(e + cells - 1) % cells], &r = speeds[e];
        double alpha = std::max({l.a, l.b, r.a, r.b});
        for (int q = 0; q < basis.points; ++q)
            alpha = std::max(alpha, example.gas.spectral_radius(quadrature_state(u, e, q)));
        rate = std::max(rate, alpha / h);
    }
    require(std::isfinite(rate) && rate > 0, "Invalid CFL rate");
    return rate;
}
// discretization.cpp:93-101
void Problem::trace(const Vec &u, Vec &lambda) const {
    lambda.assign((size_t)cells * NVAR, 0.);
    for (int f = 0; f < cells; ++f) {
        const State l = sample(u, f, basis.right), r = sample(u, (f + 1) % cells, basis.left);
        const Speed s = speeds[f];
        const State fl = example.gas.flux(l), fr = example.gas.flux(r);
        for (int v = 0; v < NVAR; ++v) lambda[f * NVAR + v] = (s.a * l[v] + s.b * r[v] + fl[v] - fr[v]) / (s.a + s.b);
    }
}
// discretization.cpp:102-112
void Problem::volume_residual(const Vec &u, Vec &r) const {
    r.assign(size(), 0.);
    for (int i = 0; i < size(); ++i) r[i] = mass[i] * (u[i] - old[i]) / step_size;
    if (n == 1) return;
    const int Q = basis.points;
    std::vector<State> flux(Q);
    for (int e = 0; e < cells; ++e) {
        for (int q = 0; q < Q; ++q) flux[q] = example.gas.flux(quadrature_state(u, e, q));
        for (int v = 0; v < NVAR; ++v)
            for (int i = 0; i < n; ++i) {
                double s = 0;
                for (int q = 0; q < Q; ++q) s += basis.wd[q * n + i] * flux[q][v];
                r[index(e, v, i)] -= s;
            }
    }
}
// discretization.cpp:113-127
void Problem::dg_residual(const Vec &u, Vec &r) const {
    volume_residual(u, r);
    for (int e = 0; e < cells; ++e) {
        const int next = (e + 1) % cells;
        const Speed s = speeds[e];
        const State l = sample(u, e, basis.right), rr = sample(u, next, basis.left);
        const State fl = example.gas.flux(l), fr = example.gas.flux(rr);
        for (int v = 0; v < NVAR; ++v) {
            const double f = (s.b * fl[v] + s.a * fr[v] + s.a * s.b * (l[v] - rr[v])) / (s.a + s.b);
            for (int i = 0; i < n; ++i) {
                r[index(e, v, i)] += basis.right[i] * f;
                r[index(next, v, i)] -= basis.left[i] * f;
            }
        }
    }
}
// discretization.cpp:128-144
bool Problem::admissible(const Vec &u) const {
    for (double x : u)
        if (!std::isfinite(x)) return false;
    auto ok = [&](const State &z) { return z[Density] > 1e-13 && example.gas.pressure(z) > 1e-13; };
    for (int e = 0; e < cells; ++e) {
        for (int i = 0; i < n; ++i)
            if (!ok({u[index(e, 0, i)], u[index(e, 1, i)], u[index(e, 2, i)]})) return false;
        for (int q = 0; q < basis.points; ++q)
            if (!ok(quadrature_state(u, e, q))) return false;
        if (!ok(sample(u, e, basis.left)) || !ok(sample(u, e, basis.right))) return false;
    }
    return true;
}
// discretization.cpp:145-147
double Problem::residual_norm(const Vec &r) const {
    double s = 0;
    for (int i = 0; i < size(); ++i) s += r[i] * r[i] * inverse_mass[i];
    return std::sqrt(.5 * s);
}
// discretization.cpp:148-155
State Problem::integral(const Vec &u) const {
    State total{0., 0., 0.};
    for (int e = 0; e < cells; ++e)
        for (int v = 0; v < NVAR; ++v)
            for (int i = 0; i < n; ++i) total[v] += .5 * h * basis.w[i] * u[index(e, v, i)];
    return total;
}
// discretization.cpp:156-168
State Problem::error(const Vec &u, double t) const {
    State squared{0., 0., 0.};
    const int Qe = (int)basis.ex.size();
    for (int e = 0; e < cells; ++e)
        for (int q = 0; q < Qe; ++q) {
            State z{0., 0., 0.};
            for (int v = 0; v < NVAR; ++v)
                for (int i = 0; i < n; ++i) z[v] += basis.evalues[q * n + i] * u[index(e, v, i)];
            const State ex = example.exact(-1 + h * (e + .5) + .5 * h * basis.ex[q], t);
            for (int v = 0; v < NVAR; ++v) squared[v] += .5 * h * basis.ew[q] * (z[v] - ex[v]) * (z[v] - ex[v]);
        }
    for (auto &s : squared) s = std::sqrt(s);
    return squared;
}

// ---------------------------------------------------------------- dg_hdg_1d/src/volume_jacobian.cpp
void VolumeJacobian::refresh(const Vec &u) {  // :17-37
    require(p_.step_size > 0, "Set the time step before refreshing the volume Jacobian");
    inverse_step_ = 1 / p_.step_size;
    ready_ = true;
    if (p_.n == 1) return;
    const int Q = p_.basis.points;
    coef_.assign((size_t)p_.cells * Q, Jac{});
    for (int cell = 0; cell < p_.cells; ++cell)
        for (int q = 0; q < Q; ++q) coef_[(size_t)cell * Q + q] = p_.example.gas.jacobian(p_.quadrature_state(u, cell, q));
}
void VolumeJacobian::apply(const Vec &d, Vec &out) const {  // :78-104
    require(ready_, "Refresh the volume Jacobian before applying it");
    const int n = p_.n, Q = p_.basis.points;
    out.assign(p_.size(), 0.);
    for (int i = 0; i < p_.size(); ++i) out[i] = p_.mass[i] * d[i] * inverse_step_;
    if (n == 1) return;
    std::vector<State> dir(Q), fd(Q);
    for (int cell = 0; cell < p_.cells; ++cell) {
        for (int q = 0; q < Q; ++q) dir[q] = p_.quadrature_state(d, cell, q);
        for (int q = 0; q < Q; ++q) {
            const Jac &J = coef_[(size_t)cell * Q + q];
            for (int v = 0; v < NVAR; ++v) {
                double s = 0;
                for (int w = 0; w < NVAR; ++w) s += J[v * NVAR + w] * dir[q][w];
                fd[q][v] = s;
            }
        }
        for (int v = 0; v < NVAR; ++v)
            for (int i = 0; i < n; ++i) {
                double s = 0;
                for (int q = 0; q < Q; ++q) s += p_.basis.wd[q * n + i] * fd[q][v];
                out[p_.index(cell, v, i)] -= s;
            }
    }
}
// :105-131 — A_(v,i),(w,j) = -sum_q wd(q,i) J_q(v,w) values(q,j), plus M / tau on the diagonal.
void VolumeJacobian::block(int cell, double *out) const {
    require(ready_, "Refresh the volume Jacobian before assembling a block");
    const int n = p_.n, Q = p_.basis.points, m = p_.block;
    std::fill(out, out + (size_t)m * m, 0.);
    if (n > 1)
        for (int w = 0; w < NVAR; ++w)
            for (int j = 0; j < n; ++j)
                for (int v = 0; v < NVAR; ++v)
                    for (int i = 0; i < n; ++i) {
                        double s = 0;
                        for (int q = 0; q < Q; ++q)
                            s += p_.basis.wd[q * n + i] * coef_[(size_t)cell * Q + q][v * NVAR + w] *
                                 p_.basis.values[q * n + j];
                        out[(size_t)p_.local(w, j) * m + p_.local(v, i)] = -s;
                    }
    for (int r = 0; r < m; ++r) out[(size_t)r * m + r] += p_.mass[(size_t)cell * m + r] * inverse_step_;
}

// ---------------------------------------------------------------- dg_hdg_1d/src/dg_operator.cpp
void DGOperator::refresh(const Vec &u) {  // :7-23
    volume_.refresh(u);
    left_.assign(p_.cells, Jac{});
    right_.assign(p_.cells, Jac{});
    for (int f = 0; f < p_.cells; ++f) {
        const int next = (f + 1) % p_.cells;
        const Speed s = p_.speeds[f];
        const Jac jl = p_.example.gas.jacobian(p_.sample(u, f, p_.basis.right));
        const Jac jr = p_.example.gas.jacobian(p_.sample(u, next, p_.basis.left));
        for (int v = 0; v < NVAR; ++v)
            for (int w = 0; w < NVAR; ++w) {
                left_[f][v * NVAR + w] = s.b / (s.a + s.b) * (jl[v * NVAR + w] + (v == w ? s.a : 0.));
                right_[f][v * NVAR + w] = s.a / (s.a + s.b) * (jr[v * NVAR + w] - (v == w ? s.b : 0.));
            }
    }
    ready_ = true;
}
void DGOperator::apply(const Vec &d, Vec &out) const {  // :24-49
    require(ready_, "Refresh the DG Jacobian before applying it");
    volume_.apply(d, out);
    for (int f = 0; f < p_.cells; ++f) {
        const int next = (f + 1) % p_.cells;
        const State l = p_.sample(d, f, p_.basis.right), r = p_.sample(d, next, p_.basis.left);
        State flux;
        for (int v = 0; v < NVAR; ++v) {
            double s = 0;
            for (int w = 0; w < NVAR; ++w) s += left_[f][v * NVAR + w] * l[w] + right_[f][v * NVAR + w] * r[w];
            flux[v] = s;
        }
        for (int v = 0; v < NVAR; ++v)
            for (int i = 0; i < p_.n; ++i) {
                out[p_.index(f, v, i)] += p_.basis.right[i] * flux[v];
                out[p_.index(next, v, i)] -= p_.basis.left[i] * flux[v];
            }
    }
}
void DGOperator::block(int row, int col, double *out) const {  // :50-78
    require(ready_, "Refresh the DG Jacobian before assembling a block");
    const int m = p_.block, n = p_.n, cells = p_.cells;
    if (row == col) volume_.block(row, out);
    else std::fill(out, out + (size_t)m * m, 0.);
    for (int side = 0; side < NFACES; ++side) {
        const int face = side == 0 ? (row + cells - 1) % cells : row, next = (face + 1) % cells;
        if (col != face && col != next) continue;
        const Vec &test = side == 0 ? p_.basis.left : p_.basis.right;
        const double sign = side == 0 ? -1.0 : 1.0;
        for (int trace_side = 0; trace_side < NFACES; ++trace_side) {
            if (col != (trace_side == 0 ? face : next)) continue;
            const Vec &trial = trace_side == 0 ? p_.basis.right : p_.basis.left;
            const Jac &D = trace_side == 0 ? left_[face] : right_[face];
            for (int w = 0; w < NVAR; ++w)
                for (int j = 0; j < n; ++j)
                    for (int v = 0; v < NVAR; ++v)
                        for (int i = 0; i < n; ++i)
                            out[(size_t)p_.local(w, j) * m + p_.local(v, i)] += sign * trial[j] * D[v * NVAR + w] * test[i];
        }
    }
}

// ---------------------------------------------------------------- dg_hdg_1d/src/hybrid.cpp
HybridOperator::HybridOperator(const Problem &p) : p_(p), volume_(p), cells_(p.cells) {}
int HybridOperator::face_index(int cell, int side) const {  // :11-13
    return side == 0 ? (cell + p_.cells - 1) % p_.cells : cell;
}
// :39-84 with the skeleton residual zero (refresh_projected).
void HybridOperator::refresh_projected(const Vec &u, const Vec &r) {
    const int m = p_.block, n = p_.n, T = NFACES * NVAR;
    volume_.refresh(u);
    rhs_.assign((size_t)p_.cells * NVAR, 0.);
    Vec A((size_t)m * m);
    for (int cell = 0; cell < p_.cells; ++cell) {
        Cell &d = cells_[cell];
        volume_.block(cell, A.data());
        d.B.assign((size_t)m * T, 0.);
        d.C.assign((size_t)T * m, 0.);
        for (int side = 0; side < NFACES; ++side) {
            const Speed s = p_.speeds[face_index(cell, side)];
            const Vec &shape = side == 0 ? p_.basis.left : p_.basis.right;
            const double sign = side == 0 ? -1.0 : 1.0, stab = side == 0 ? s.b : s.a;
            const Jac J = p_.example.gas.jacobian(p_.sample(u, cell, shape));
            Jac deriv;
            for (int v = 0; v < NVAR; ++v)
                for (int w = 0; w < NVAR; ++w) deriv[v * NVAR + w] = sign * J[v * NVAR + w] + (v == w ? stab : 0.);
            for (int v = 0; v < NVAR; ++v)
                for (int i = 0; i < n; ++i) {
                    const int row = p_.local(v, i);
                    d.B[(size_t)(side * NVAR + v) * m + row] = -shape[i] * stab;
                    for (int w = 0; w < NVAR; ++w) {
                        d.C[(size_t)row * T + side * NVAR + w] = shape[i] * deriv[w * NVAR + v];
                        for (int j = 0; j < n; ++j)
                            A[(size_t)p_.local(w, j) * m + row] += shape[i] * shape[j] * deriv[v * NVAR + w];
                    }
                }
        }
        oracle::DenseLU lu;
        lu.compute(A.data(), m);
        d.X.assign((size_t)m * T, 0.);
        for (int j = 0; j < T; ++j) lu.solve(&d.B[(size_t)j * m], &d.X[(size_t)j * m]);
        d.y.assign(m, 0.);
        lu.solve(&r[(size_t)cell * m], d.y.data());
        d.S.assign((size_t)T * T, 0.);
        for (int j = 0; j < T; ++j)
            for (int a = 0; a < T; ++a) {
                double s = 0;
                for (int k = 0; k < m; ++k) s += d.C[(size_t)k * T + a] * d.X[(size_t)j * m + k];
                d.S[(size_t)j * T + a] = -s;
            }
        for (int side = 0; side < NFACES; ++side)
            for (int v = 0; v < NVAR; ++v) {
                double s = 0;
                for (int k = 0; k < m; ++k) s += d.C[(size_t)k * T + side * NVAR + v] * d.y[k];
                rhs_[(size_t)face_index(cell, side) * NVAR + v] += s;
            }
    }
}
void HybridOperator::apply(const Vec &x, Vec &y) const {  // :85-103
    const int T = NFACES * NVAR;
    y.assign((size_t)p_.cells * NVAR, 0.);
    for (int f = 0; f < p_.cells; ++f)
        for (int v = 0; v < NVAR; ++v) y[(size_t)f * NVAR + v] = -(p_.speeds[f].a + p_.speeds[f].b) * x[(size_t)f * NVAR + v];
    double g[T];
    for (int cell = 0; cell < p_.cells; ++cell) {
        for (int side = 0; side < NFACES; ++side)
            for (int v = 0; v < NVAR; ++v) g[side * NVAR + v] = x[(size_t)face_index(cell, side) * NVAR + v];
        for (int a = 0; a < T; ++a) {
            double s = 0;
            for (int j = 0; j < T; ++j) s += cells_[cell].S[(size_t)j * T + a] * g[j];
            y[(size_t)face_index(cell, a / NVAR) * NVAR + a % NVAR] += s;
        }
    }
}
void HybridOperator::block(int row, int col, double *out) const {  // :104-117
    const int T = NFACES * NVAR;
    std::fill(out, out + NVAR * NVAR, 0.);
    if (row == col)
        for (int v = 0; v < NVAR; ++v) out[v * NVAR + v] = -(p_.speeds[row].a + p_.speeds[row].b);
    for (int adjacent = 0; adjacent < NFACES; ++adjacent) {
        const int cell = (row + adjacent) % p_.cells, row_side = adjacent == 0 ? 1 : 0;
        for (int col_side = 0; col_side < NFACES; ++col_side)
            if (face_index(cell, col_side) == col)
                for (int w = 0; w < NVAR; ++w)
                    for (int v = 0; v < NVAR; ++v)
                        out[w * NVAR + v] += cells_[cell].S[(size_t)(col_side * NVAR + w) * T + row_side * NVAR + v];
    }
}
void HybridOperator::recovered_residual(const Vec &dl, Vec &out) const {  // :118-130
    const int m = p_.block, T = NFACES * NVAR;
    Vec e;
    apply(dl, e);
    for (size_t i = 0; i < e.size(); ++i) e[i] -= rhs_[i];
    out.assign(p_.size(), 0.);
    double g[T];
    for (int cell = 0; cell < p_.cells; ++cell) {
        for (int side = 0; side < NFACES; ++side) {
            const int f = face_index(cell, side);
            const Speed s = p_.speeds[f];
            for (int v = 0; v < NVAR; ++v) g[side * NVAR + v] = e[(size_t)f * NVAR + v] / -(s.a + s.b);
        }
        for (int r = 0; r < m; ++r) {
            double s = 0;
            for (int j = 0; j < T; ++j) s += cells_[cell].B[(size_t)j * m + r] * g[j];
            out[(size_t)cell * m + r] = -s;
        }
    }
}
void HybridOperator::recover(const Vec &dl, Vec &du) const {  // :131-138
    const int m = p_.block, T = NFACES * NVAR;
    du.assign(p_.size(), 0.);
    double g[T];
    for (int cell = 0; cell < p_.cells; ++cell) {
        for (int side = 0; side < NFACES; ++side)
            for (int v = 0; v < NVAR; ++v) g[side * NVAR + v] = dl[(size_t)face_index(cell, side) * NVAR + v];
        for (int r = 0; r < m; ++r) {
            double s = 0;
            for (int j = 0; j < T; ++j) s += cells_[cell].X[(size_t)j * m + r] * g[j];
            du[(size_t)cell * m + r] = -cells_[cell].y[r] - s;
        }
    }
}

// ---------------------------------------------------------------- dg_hdg_1d/src/time_integrator.cpp:45-206
namespace {
using Clock = std::chrono::steady_clock;
double elapsed(Clock::time_point s) { return std::chrono::duration<double>(Clock::now() - s).count(); }
template <class Op> void bind_apply(const void *c, const Vec &x, Vec &y) { static_cast<const Op *>(c)->apply(x, y); }
// The block-Jacobi kind of BlockPreconditioner (common/src/linalg/block_ilu.cpp:48-84): one
// DenseLU per diagonal block, whose own require() messages report a failure.
struct Jacobi {
    int blocks, width;
    std::vector<oracle::DenseLU> lus;
    Jacobi(int b, int w) : blocks(b), width(w), lus(b) {}
    template <class F> void refresh(F &&provider) {
        Vec blk((size_t)width * width);
        for (int i = 0; i < blocks; ++i) {
            provider(i, i, blk.data());
            lus[i].compute(blk.data(), width);
        }
    }
    void apply(const Vec &rhs, Vec &out) const {
        out.resize(rhs.size());
        for (int i = 0; i < blocks; ++i) lus[i].solve(&rhs[(size_t)i * width], &out[(size_t)i * width]);
    }
};
// BlockPreconditioner on BlockGraph::periodic(cells) (dg_hdg_1d/src/time_integrator.cpp:31-36):
// block Jacobi or block ILU(0) in the natural ordering.
struct Precond1D {
    Jacobi jacobi;
    std::unique_ptr<oracle::BlockILU0> ilu;
    Precond1D(int blocks, int width, bool use_ilu) : jacobi(blocks, width) {
        if (use_ilu) ilu = std::make_unique<oracle::BlockILU0>(oracle::periodic_adjacency(blocks), width);
    }
    template <class F> void refresh(F &&provider) {
        if (ilu) ilu->refresh(provider);
        else jacobi.refresh(provider);
    }
    void apply(const Vec &rhs, Vec &out) const {
        if (ilu) ilu->apply(rhs, out);
        else jacobi.apply(rhs, out);
    }
};
}  // namespace

oracle::RunStatistics advance(Problem &p, Method method, Vec &solution) {
    const Config &c = p.config;
    const int N = p.size(), NT = p.cells * NVAR;
    const bool dg = method == Method::DG;
    require(!c.direct, "The dense direct solve is not restated in the oracle");
    require(!(c.ilu && c.colamd), "The block COLAMD ordering is not restated in the oracle");
    Vec state(N), trial(N), residual(N), trial_residual(N), direction(N), rhs(dg ? N : NT);
    Vec trace_direction(NT), equation_error(N), independent(N), step_state(N), stage_base(N);
    std::vector<Vec> slopes(4, Vec(N));
    const Vec weights = dg ? p.inverse_mass : Vec(NT, 1.);
    std::unique_ptr<DGOperator> dgop, diagnostic;
    std::unique_ptr<HybridOperator> hybrid;
    if (dg) dgop = std::make_unique<DGOperator>(p);
    else hybrid = std::make_unique<HybridOperator>(p);
    if (!dg && c.check_update) diagnostic = std::make_unique<DGOperator>(p);
    Precond1D precond(p.cells, dg ? p.block : NVAR, c.ilu);
    oracle::GMRES gmres(dg ? N : NT, c.restart, weights);
    auto dual_norm = [&](const Vec &x) {
        double s = 0;
        for (int i = 0; i < N; ++i) s += x[i] * x[i] * p.inverse_mass[i];
        return std::sqrt(s);
    };
    auto state_norm = [&](const Vec &x) {
        double s = 0;
        for (int i = 0; i < N; ++i) s += x[i] * x[i] * p.mass[i];
        return std::sqrt(s);
    };
    require((int)solution.size() == N && p.admissible(solution), "Invalid initial solution");
    require(c.steps > 0 || c.final_time < p.example.shock_time(), "Final time reaches simple-wave shock");
    constexpr double alpha = .24169426078821, beta = alpha / 4., eta = .12915286960590;
    constexpr double a[4][4] = {{alpha, 0, 0, 0}, {-alpha, alpha, 0, 0}, {0, 1 - alpha, alpha, 0},
                                {beta, eta, .5 - beta - eta - alpha, alpha}};
    constexpr double b[4] = {0, 1. / 6, 1. / 6, 2. / 3}, stage_c[4] = {alpha, 0, 1, .5};
    const int stages = c.integrator == "be" ? 1 : 4;
    oracle::RunStatistics stats;
    p.freeze(solution);
    const State initial_integral = p.integral(solution);
    const auto begin = Clock::now();
    while (c.steps > 0 ? stats.steps < c.steps : stats.final_time < c.final_time) {
        const double rate = p.freeze(solution);
        double step = c.cfl / rate;
        if (c.steps == 0) {
            const double remaining = c.final_time - stats.final_time;
            step = std::min(step, remaining);
            if (remaining - step <= 16 * std::numeric_limits<double>::epsilon() * std::max(remaining, c.final_time))
                step = remaining;
        }
        require(std::isfinite(step) && step > 0 && stats.final_time + step > stats.final_time, "Invalid CFL step");
        require(stats.final_time + step < p.example.shock_time(), "Step reaches simple-wave shock");
        step_state = solution;
        state = solution;
        for (int stage = 0; stage < stages; ++stage) {
            const double diagonal = stages == 1 ? 1. : a[stage][stage];
            stage_base = step_state;
            for (int j = 0; j < stage; ++j)
                for (int i = 0; i < N; ++i) stage_base[i] += step * a[stage][j] * slopes[j][i];
            if (stage > 0) p.freeze(state);
            p.step_size = diagonal * step;
            p.old = stage_base;
            const double tau = p.step_size, old_norm = state_norm(stage_base);
            const int limit = c.newton_steps > 0 ? c.newton_steps : c.max_newton;
            double initial_rms = -1.;
            bool converged = false, residual_ready = false;
            for (int it = 0; it <= limit; ++it) {
                const auto update_start = Clock::now();
                if (!residual_ready) p.dg_residual(state, residual);
                const double norm = dual_norm(residual), rms = norm / std::sqrt(2.);
                if (initial_rms < 0) initial_rms = rms;
                if (c.newton_steps == 0 && rms <= c.nonlinear_tolerance * std::max(1., initial_rms)) {
                    converged = true;
                    break;
                }
                if (it == limit) break;
                const double allowance = 128 * std::numeric_limits<double>::epsilon() *
                                         ((state_norm(state) + old_norm) / tau + norm);
                const double target = std::max(10 * c.linear_tolerance * norm, allowance);
                oracle::LinearResult linear{0, 0};
                if (dg) {
                    dgop->refresh(state);
                    for (int i = 0; i < N; ++i) rhs[i] = -residual[i];
                    precond.refresh([&](int row, int col, double *out) { dgop->block(row, col, out); });
                    linear = gmres.solve(oracle::Action{dgop.get(), bind_apply<DGOperator>},
                                         oracle::Action{&precond, bind_apply<Precond1D>}, rhs, direction, c.max_linear,
                                         c.linear_tolerance);
                    for (int i = 0; i < N; ++i) equation_error[i] = -gmres.residual()[i];
                } else {
                    hybrid->refresh_projected(state, residual);
                    rhs = hybrid->rhs();
                    precond.refresh([&](int row, int col, double *out) { hybrid->block(row, col, out); });
                    double tolerance = c.linear_tolerance;
                    bool valid = false;
                    for (int attempt = 0; attempt < 4; ++attempt) {
                        const oracle::LinearResult cur =
                            gmres.solve(oracle::Action{hybrid.get(), bind_apply<HybridOperator>},
                                        oracle::Action{&precond, bind_apply<Precond1D>}, rhs, trace_direction,
                                        c.max_linear, tolerance);
                        linear.iterations += cur.iterations;
                        linear.relative_residual = cur.relative_residual;
                        hybrid->recover(trace_direction, direction);
                        hybrid->recovered_residual(trace_direction, equation_error);
                        valid = dual_norm(equation_error) <= target;
                        if (valid) break;
                        tolerance *= .01;
                    }
                    require(valid, "Recovered DG residual criterion failed after Schur refinement");
                }
                const double error_norm = dual_norm(equation_error);
                require(error_norm <= target, "DG Newton linear residual too large");
                if (diagnostic) {
                    diagnostic->refresh(state);
                    diagnostic->apply(direction, independent);
                    for (int i = 0; i < N; ++i) independent[i] += residual[i];
                    require(dual_norm(independent) <= std::max(4 * target, 1e-12),
                            "Independent recovered DG equation check failed");
                    for (int i = 0; i < N; ++i) independent[i] -= equation_error[i];
                    require(dual_norm(independent) <= std::max(4 * allowance, 1e-12),
                            "Recovered residual identity failed");
                }
                double damping = 1.;
                bool accepted = false;
                for (int search = 0; search < 30; ++search) {
                    for (int i = 0; i < N; ++i) trial[i] = state[i] + damping * direction[i];
                    if (p.admissible(trial)) {
                        p.dg_residual(trial, trial_residual);
                        if (dual_norm(trial_residual) <= (1 - 1e-4 * damping) * norm + allowance) {
                            accepted = true;
                            break;
                        }
                    }
                    damping *= .5;
                }
                require(accepted, "Newton line search failed");
                state.swap(trial);
                residual.swap(trial_residual);
                residual_ready = true;
                const double duration = elapsed(update_start);
                stats.max_linear_residual = std::max(stats.max_linear_residual, linear.relative_residual);
                const double dgrel = norm > 0 ? error_norm / norm : 0.;
                stats.max_dg_linear_residual = std::max(stats.max_dg_linear_residual, dgrel);
                stats.krylov_iterations += linear.iterations;
                if (stats.newton_iterations >= c.warmup_updates) {
                    stats.measured_newton_seconds += duration;
                    ++stats.measured_updates;
                }
                ++stats.newton_iterations;
                stats.updates.push_back({stats.steps, stage, it, linear.iterations, stats.final_time + step,
                                         stats.final_time + (stages == 1 ? 1. : stage_c[stage]) * step, step,
                                         step * rate, rms, damping, linear.relative_residual, dgrel, duration});
            }
            require(converged || c.newton_steps > 0, "Newton iteration limit reached");
            for (int i = 0; i < N; ++i) slopes[stage][i] = (state[i] - stage_base[i]) / tau;
        }
        if (stages == 1) solution = state;
        else {
            solution = step_state;
            for (int s = 0; s < stages; ++s)
                for (int i = 0; i < N; ++i) solution[i] += step * b[s] * slopes[s][i];
            require(p.admissible(solution), "DIRK3 step produced an inadmissible state");
        }
        stats.final_time = c.steps == 0 && step >= c.final_time - stats.final_time ? c.final_time
                                                                                   : stats.final_time + step;
        stats.minimum_step = stats.steps == 0 ? step : std::min(stats.minimum_step, step);
        stats.maximum_step = std::max(stats.maximum_step, step);
        ++stats.steps;
        const State now = p.integral(solution);
        double drift = 0;
        for (int v = 0; v < NVAR; ++v) drift = std::max(drift, std::abs(now[v] - initial_integral[v]));
        stats.conservation_drift = std::max(stats.conservation_drift, drift);
    }
    stats.seconds = elapsed(begin);
    return stats;
}

// ---------------------------------------------------------------- dg_hdg_1d/src/main.cpp:7-107
int run_main(int argc, char **argv) {
    try {
        const Config config = parse(argc, argv);
        Problem problem(config);
        {
            const std::string &prefix = config.prefix;
            std::string accum;
            const auto slash = prefix.find_last_of('/');
            if (slash != std::string::npos)
                for (size_t i = 0; i <= slash; ++i) {
                    if (i == slash || prefix[i] == '/') {
                        if (!accum.empty()) mkdir(accum.c_str(), 0755);
                    }
                    accum += prefix[i];
                }
        }
        std::ofstream summary(config.prefix + "_summary.csv"), updates(config.prefix + "_iterations.csv");
        require(bool(summary) && bool(updates), "Cannot open output files");
        summary << std::setprecision(17)
                << "method,cells,k,quad,cfl,integrator,linear,preconditioner,ordering,ntol,ltol,safety,"
                   "fixed_newton_steps,warmup_updates,steps,final_time,newton_iterations,krylov_iterations,"
                   "max_linear_relative_residual,max_dg_linear_relative_residual,min_step,max_step,mean_dt,"
                   "time_loop_s,measured_updates,mean_newton_s,volume_dofs,trace_dofs,"
                   "rho_L2,momentum_L2,energy_L2,max_conservation_drift\n";
        updates << std::setprecision(17)
                << "method,step,stage,iteration,time,stage_time,dt,cfl,residual_physical_rms,damping,"
                   "krylov_iterations,linear_relative_residual,dg_linear_relative_residual,iteration_s,measured\n";
        std::ofstream solution_file;
        if (!config.timing_only) {
            solution_file.open(config.prefix + "_solution.csv");
            require(bool(solution_file), "Cannot open solution output");
            solution_file << std::setprecision(17)
                          << "method,cell,node,x,rho,momentum,energy,rho_exact,momentum_exact,energy_exact\n";
        }
        Vec dg_solution, solution;
        bool have_dg = false;
        for (Method method : {Method::DG, Method::HDG}) {
            const std::string name = method == Method::DG ? "dg" : "hdg";
            if (config.method != "both" && config.method != name) continue;
            problem.initial(solution);
            const auto stats = advance(problem, method, solution);
            State error;
            if (config.timing_only) error.fill(std::numeric_limits<double>::quiet_NaN());
            else error = problem.error(solution, stats.final_time);
            summary << name << ',' << config.cells << ',' << config.degree << ',' << problem.basis.points << ','
                    << config.cfl << ',' << config.integrator << ',' << (config.direct ? "direct" : "gmres") << ','
                    << (config.direct ? "none" : config.ilu ? "block-ilu0" : "block-jacobi") << ','
                    << (config.direct ? "none" : !config.ilu || !config.colamd ? "natural" : "colamd") << ','
                    << config.nonlinear_tolerance << ',' << config.linear_tolerance << ',' << config.safety << ','
                    << config.newton_steps << ',' << config.warmup_updates << ',' << stats.steps << ','
                    << stats.final_time << ',' << stats.newton_iterations << ',' << stats.krylov_iterations << ','
                    << stats.max_linear_residual << ',' << stats.max_dg_linear_residual << ','
                    << stats.minimum_step << ',' << stats.maximum_step << ','
                    << (stats.steps ? stats.final_time / stats.steps : 0.) << ',' << stats.seconds << ','
                    << stats.measured_updates << ','
                    << (stats.measured_updates ? stats.measured_newton_seconds / stats.measured_updates : 0.)
                    << ',' << problem.size() << ',' << problem.cells * NVAR;
            for (int v = 0; v < NVAR; ++v) summary << ',' << error[v];
            summary << ',' << stats.conservation_drift << '\n';
            for (size_t i = 0; i < stats.updates.size(); ++i) {
                const auto &u = stats.updates[i];
                updates << name << ',' << u.step << ',' << u.stage << ',' << u.iteration << ',' << u.time << ','
                        << u.stage_time << ',' << u.dt << ',' << u.cfl << ',' << u.residual_physical_rms << ','
                        << u.damping << ',' << u.krylov_iterations << ',' << u.linear_relative_residual << ','
                        << u.dg_linear_relative_residual << ',' << u.iteration_s << ','
                        << (i >= static_cast<size_t>(config.warmup_updates)) << '\n';
            }
            if (!config.timing_only)
                for (int cell = 0; cell < problem.cells; ++cell)
                    for (int i = 0; i < problem.n; ++i) {
                        const double x = -1 + problem.h * (cell + .5) + .5 * problem.h * problem.basis.x[i];
                        const State exact = problem.example.exact(x, stats.final_time);
                        solution_file << name << ',' << cell << ',' << i << ',' << x;
                        for (int v = 0; v < NVAR; ++v) solution_file << ',' << solution[problem.index(cell, v, i)];
                        for (int v = 0; v < NVAR; ++v) solution_file << ',' << exact[v];
                        solution_file << '\n';
                    }
            std::cout << name << ": steps=" << stats.steps << ", Newton=" << stats.newton_iterations
                      << ", Krylov=" << stats.krylov_iterations << ", time=" << stats.seconds << " s, mean Newton="
                      << (stats.measured_updates ? stats.measured_newton_seconds / stats.measured_updates : 0.)
                      << " s, conservation drift=" << stats.conservation_drift << '\n';
            if (method == Method::DG) {
                dg_solution = solution;
                have_dg = true;
            } else if (have_dg) {
                double maximum = 0;
                for (int i = 0; i < problem.size(); ++i)
                    maximum = std::max(maximum, std::abs(dg_solution[i] - solution[i]));
                std::ofstream comparison(config.prefix + "_difference.csv");
                require(bool(comparison), "Cannot open comparison output");
                comparison << std::setprecision(17) << "rho_L2,momentum_L2,energy_L2,joint_L2,max_nodal\n";
                double joint = 0.;
                for (int v = 0; v < NVAR; ++v) {
                    double squared = 0.;
                    for (int cell = 0; cell < problem.cells; ++cell)
                        for (int i = 0; i < problem.n; ++i) {
                            const int k = problem.index(cell, v, i);
                            const double d = dg_solution[k] - solution[k];
                            squared += d * d * problem.mass[k];
                        }
                    comparison << std::sqrt(squared) << ',';
                    joint += squared;
                }
                comparison << std::sqrt(joint) << ',' << maximum << '\n';
                std::cout << "DG/HDG max difference=" << maximum << '\n';
                require(maximum < 1e-8, "DG/HDG solutions disagree");
            }
        }
    } catch (const std::exception &error) {
        std::cerr << "ERROR: " << error.what() << '\n';
        return 1;
    }
    return 0;
}
}  // namespace oracle1d
