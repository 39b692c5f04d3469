// Test infrastructure only: CPU oracle for the 2D DG / condensed-HDG Euler Newton update.
// A plain C++17 restatement of YueWu2002/DG_HDG_Euler_Cpp (dg_hdg_2d/src, common/) without
// Eigen.  Used by tests/, the smoke check and the cpu_baseline leg of bench.py only; the
// product library never links it.  See dgh_oracle.hpp for the interface.
#include "dgh_oracle.hpp"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <sys/stat.h>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace oracle {

void set_threads(int threads) {
#ifdef _OPENMP
    omp_set_num_threads(threads > 0 ? threads : 1);
#else
    (void)threads;
#endif
}

// ---------------------------------------------------------------- config.cpp:6-122
void validate(const Config &c) {
    require(c.nx >= 3 && c.ny >= 3 && c.degree >= 0 && c.degree <= 8 && c.quadrature >= 0,
            "Invalid mesh or degree");
    require(c.testcase == "diagonal" || c.testcase == "wave" || c.testcase == "axis",
            "Invalid testcase");
    require(c.quadrature == 0 || c.quadrature >= c.degree + 1, "Quadrature must be >= degree+1");
    require(c.restart > 0 && c.max_linear > 0 && c.max_newton > 0 && c.steps >= 0,
            "Invalid iteration limit");
    require(c.newton_steps >= 0 && c.warmup_updates >= 0, "Invalid timing update count");
    require(c.integrator == "be" || c.integrator == "ssp-dirk3", "Invalid integrator");
    require(std::isfinite(c.cfl) && c.cfl > 0 && std::isfinite(c.final_time) && c.final_time >= 0,
            "CFL must be positive and final time nonnegative");
    require(std::isfinite(c.safety) && c.safety >= 1 && std::isfinite(c.nonlinear_tolerance) &&
                c.nonlinear_tolerance > 0 && std::isfinite(c.linear_tolerance) &&
                c.linear_tolerance > 0 && c.linear_tolerance < 1,
            "Invalid solver tolerance or wave-speed safety");
    require(c.method == "dg" || c.method == "hdg" || c.method == "both",
            "Method must be dg, hdg, or both");
}

Config parse(int argc, char **argv) {
    Config c;
    bool time_seen = false, steps_seen = false;
    for (int i = 1; i < argc; ++i) {
        std::string option = argv[i];
        auto value = [&]() {
            require(i + 1 < argc, "Missing option value");
            return std::string(argv[++i]);
        };
        auto integer = [&]() {
            auto text = value();
            std::size_t end;
            int n = std::stoi(text, &end);
            require(end == text.size(), "Invalid integer");
            return n;
        };
        auto real = [&]() {
            auto text = value();
            std::size_t end;
            double n = std::stod(text, &end);
            require(end == text.size(), "Invalid number");
            return n;
        };
        if (option == "--nx") c.nx = integer();
        else if (option == "--ny") c.ny = integer();
        else if (option == "--testcase") c.testcase = value();
        else if (option == "--no-save-solution") c.save_solution = false;
        else if (option == "--newton-steps") c.newton_steps = integer();
        else if (option == "--warmup-updates") c.warmup_updates = integer();
        else if (option == "--integrator") c.integrator = value();
        else if (option == "--timing-only") c.timing_only = true;
        else if (option == "--check-update") c.check_update = true;
        else if (option == "--k") c.degree = integer();
        else if (option == "--quad") c.quadrature = integer();
        else if (option == "--cfl") c.cfl = real();
        else if (option == "--T") { c.final_time = real(); time_seen = true; }
        else if (option == "--steps") { c.steps = integer(); steps_seen = true; }
        else if (option == "--safety") c.safety = real();
        else if (option == "--method") c.method = value();
        else if (option == "--prefix") c.prefix = value();
        else if (option == "--ntol") c.nonlinear_tolerance = real();
        else if (option == "--ltol") c.linear_tolerance = real();
        else if (option == "--restart") c.restart = integer();
        else if (option == "--max-linear") c.max_linear = integer();
        else if (option == "--max-newton") c.max_newton = integer();
        else if (option == "--threads") set_threads(integer());
        else if (option == "--linear") {
            auto name = value();
            require(name == "direct" || name == "gmres", "Invalid linear solver");
            c.direct = name == "direct";
        } else if (option == "--ordering") {
            auto order = value();
            require(order == "natural" || order == "colamd", "Invalid ordering");
            c.colamd = order == "colamd";
        } else if (option == "--precond") {
            auto name = value();
            require(name == "block-jacobi", "2D currently supports block-jacobi only");
        } else throw std::runtime_error("Unknown option: " + option);
    }
    require(!(time_seen && steps_seen), "Choose either --T or --steps");
    require(!steps_seen || c.steps > 0, "steps must be positive");
    validate(c);
    return c;
}

// ---------------------------------------------------------------- nodal_basis.hpp:12-66
// Gauss-Legendre rule by Newton's method on P_n (the reference uses Bogaert's fastgl;
// both are accurate to a few ulps).  Ascending nodes, the middle node exactly 0 for odd n.
void gauss(int n, Vec &x, Vec &w) {
    require(n > 0, "Gauss rule requires a positive point count");
    x.assign(n, 0.);
    w.assign(n, 0.);
    const double pi = std::acos(-1.);
    for (int k = 0; k < (n + 1) / 2; ++k) {
        long double z = std::cos(pi * (k + .75) / (n + .5));
        long double dp = 1;
        for (int it = 0; it < 100; ++it) {
            long double p0 = 1, p1 = z;
            for (int j = 2; j <= n; ++j) {
                long double p2 = ((2 * j - 1) * z * p1 - (j - 1) * p0) / j;
                p0 = p1;
                p1 = p2;
            }
            if (n == 1) { p1 = z; p0 = 1; }
            dp = n * (z * p1 - p0) / (z * z - 1);
            long double dz = p1 / dp;
            z -= dz;
            if (std::fabs((double)dz) <= 1e-19L) break;
        }
        long double p0 = 1, p1 = z;
        for (int j = 2; j <= n; ++j) {
            long double p2 = ((2 * j - 1) * z * p1 - (j - 1) * p0) / j;
            p0 = p1;
            p1 = p2;
        }
        if (n == 1) { p1 = z; p0 = 1; }
        dp = n * (z * p1 - p0) / (z * z - 1);
        double weight = (double)(2 / ((1 - z * z) * dp * dp));
        x[n - 1 - k] = (double)z;
        x[k] = -(double)z;
        w[k] = w[n - 1 - k] = weight;
    }
    if (n % 2) x[n / 2] = 0;
}

Vec Basis::evaluate(double z) const {
    Vec v(nodes, 1.);
    for (int i = 0; i < nodes; ++i)
        for (int j = 0; j < nodes; ++j)
            if (i != j) v[i] *= (z - x[j]) / (x[i] - x[j]);
    return v;
}

Basis::Basis(int degree, int quadrature) : nodes(degree + 1), points(quadrature ? quadrature : degree + 1) {
    const int n = nodes;
    gauss(n, x, w);
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
    dw.assign(n * n, 0.);
    for (int q = 0; q < n; ++q)
        for (int i = 0; i < n; ++i) dw[q * n + i] = w[q] * D[q * n + i];
    // nodal_basis.hpp:37-57: values at the volume points (the identity when collocated) and
    // weighted_derivatives = diag(qw) * values * D
    const int P = points;
    gauss(P, qx, qw);
    values.assign(P * n, 0.);
    for (int q = 0; q < P; ++q) {
        Vec v = evaluate(qx[q]);
        for (int i = 0; i < n; ++i) values[q * n + i] = P == n ? (q == i ? 1. : 0.) : v[i];
    }
    wd.assign(P * n, 0.);
    for (int q = 0; q < P; ++q)
        for (int i = 0; i < n; ++i) {
            double s = 0;
            for (int k = 0; k < n; ++k) s += values[q * n + k] * D[k * n + i];
            wd[q * n + i] = qw[q] * s;
        }
    left = evaluate(-1);
    right = evaluate(1);
    gauss(std::max(20, 2 * n + 3), ex, ew);
    const int Q = (int)ex.size();
    evalues.assign(Q * n, 0.);
    for (int q = 0; q < Q; ++q) {
        Vec v = evaluate(ex[q]);
        for (int i = 0; i < n; ++i) evalues[q * n + i] = v[i];
    }
    projection.assign(n * Q, 0.);
    for (int i = 0; i < n; ++i)
        for (int q = 0; q < Q; ++q) projection[i * Q + q] = evalues[q * n + i] * ew[q] / w[i];
}

// ---------------------------------------------------------------- physics.cpp:4-70
double Gas::pressure(const State &u) const {
    return (gamma - 1) *
           (u[Energy] - .5 * (u[MomentumX] * u[MomentumX] + u[MomentumY] * u[MomentumY]) / u[Density]);
}
void Gas::primitive(const State &u, double &ir, double &vx, double &vy, double &p, double &H) const {
    ir = 1 / u[Density];
    vx = u[MomentumX] * ir;
    vy = u[MomentumY] * ir;
    p = (gamma - 1) * (u[Energy] - .5 * (u[MomentumX] * vx + u[MomentumY] * vy));
    H = (u[Energy] + p) * ir;
}
State Gas::flux(const State &u, int axis) const {
    double ir, vx, vy, p, H;
    primitive(u, ir, vx, vy, p, H);
    const double va = axis == 0 ? vx : vy;
    State f;
    f[Density] = u[MomentumX + axis];
    f[MomentumX] = u[MomentumX] * va;
    f[MomentumY] = u[MomentumY] * va;
    f[MomentumX + axis] += p;
    f[Energy] = (u[Energy] + p) * va;
    return f;
}
Jac Gas::cached_jacobian(double u, double v, double H, int axis) const {
    const double gm = gamma - 1., s2 = u * u + v * v;
    Jac a{};
    if (axis == 0) {
        a[0 * 4 + 1] = 1.;
        a[1 * 4 + 0] = .5 * (gamma - 3) * u * u + .5 * gm * v * v;
        a[1 * 4 + 1] = (3 - gamma) * u;
        a[1 * 4 + 2] = -gm * v;
        a[1 * 4 + 3] = gm;
        a[2 * 4 + 0] = -u * v; a[2 * 4 + 1] = v; a[2 * 4 + 2] = u; a[2 * 4 + 3] = 0.;
        a[3 * 4 + 0] = u * (.5 * gm * s2 - H);
        a[3 * 4 + 1] = H - gm * u * u;
        a[3 * 4 + 2] = -gm * u * v;
        a[3 * 4 + 3] = gamma * u;
    } else {
        a[0 * 4 + 2] = 1.;
        a[1 * 4 + 0] = -u * v; a[1 * 4 + 1] = v; a[1 * 4 + 2] = u; a[1 * 4 + 3] = 0.;
        a[2 * 4 + 0] = .5 * gm * u * u + .5 * (gamma - 3) * v * v;
        a[2 * 4 + 1] = -gm * u;
        a[2 * 4 + 2] = (3 - gamma) * v;
        a[2 * 4 + 3] = gm;
        a[3 * 4 + 0] = v * (.5 * gm * s2 - H);
        a[3 * 4 + 1] = -gm * u * v;
        a[3 * 4 + 2] = H - gm * v * v;
        a[3 * 4 + 3] = gamma * v;
    }
    return a;
}
Speed einfeldt(const State &l, const State &r, const Gas &gas, double safety, int axis) {
    double il, ulx, uly, pl, Hl, irr, urx, ury, pr, Hr;
    gas.primitive(l, il, ulx, uly, pl, Hl);
    gas.primitive(r, irr, urx, ury, pr, Hr);
    require(l[Density] > 0 && r[Density] > 0 && pl > 0 && pr > 0, "Invalid frozen face state");
    const double sl = std::sqrt(l[Density]), sr = std::sqrt(r[Density]);
    const double vx = (sl * ulx + sr * urx) / (sl + sr), vy = (sl * uly + sr * ury) / (sl + sr);
    const double H = (sl * Hl + sr * Hr) / (sl + sr);
    const double sound = std::sqrt((gas.gamma - 1) * (H - .5 * (vx * vx + vy * vy)));
    const double cl = std::sqrt(gas.gamma * pl * il), cr = std::sqrt(gas.gamma * pr * irr);
    const double vla = axis == 0 ? ulx : uly, vra = axis == 0 ? urx : ury, va = axis == 0 ? vx : vy;
    return {safety * std::max({0., -vla + cl, -va + sound}),
            safety * std::max({0., vra + cr, va + sound})};
}

// ---------------------------------------------------------------- example.cpp:4-39
Example::Example(const std::string &name, double degrees)
    : testcase(name), cosine(std::cos(degrees * std::acos(-1.) / 180.)),
      sine(std::sin(degrees * std::acos(-1.) / 180.)),
      lx(testcase == "diagonal" ? 2. / cosine : 2.), ly(testcase == "diagonal" ? 2. / sine : 2.) {}
double Example::shock_time() const {
    if (testcase == "wave") return std::numeric_limits<double>::infinity();
    return 4 / ((gas.gamma + 1) * std::acos(-1.));
}
State Example::exact(double x, double y, double t) const {
    const double g = gas.gamma, pi = std::acos(-1.);
    State u;
    if (testcase == "wave") {
        double rho = 1 + .2 * std::sin(pi * (x - t)) * std::sin(pi * (y - .5 * t));
        u = {rho, rho, .5 * rho, 1 / (g - 1) + .625 * rho};
        return u;
    }
    require(t < shock_time(), "Simple wave reaches shock time");
    const bool diagonal = testcase == "diagonal";
    if (diagonal) x = cosine * x + sine * y;
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
    u[Density] = rho;
    u[MomentumX] = rho * velocity * (diagonal ? cosine : 1.);
    u[MomentumY] = diagonal ? rho * velocity * sine : 0.;
    u[Energy] = std::pow(rho, g) / (g - 1) + .5 * rho * velocity * velocity;
    return u;
}

// ---------------------------------------------------------------- discretization.cpp
Problem::Problem(const Config &c)
    : config(c), basis(c.degree, c.quadrature), nx(c.nx), ny(c.ny), n(basis.nodes), cells(c.nx * c.ny),
      plane(n * n), block(NVAR * n * n), example(c.testcase), hx(example.lx / c.nx),
      hy(example.ly / c.ny) {
    validate(c);
    old.assign(size(), 0.);
    mass.assign(size(), 0.);
    for (int cell = 0; cell < cells; ++cell)
        for (int v = 0; v < NVAR; ++v)
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i)
                    mass[index(cell, v, i + n * j)] = .25 * hx * hy * basis.w[i] * basis.w[j];
    trace_mass.assign(trace_size(), 0.);
    for (int f = 0; f < face_count(); ++f)
        for (int v = 0; v < NVAR; ++v)
            for (int q = 0; q < n; ++q) trace_mass[f * face_width() + v * n + q] = face_weight(f, q);
    inverse_mass.resize(mass.size());
    for (size_t i = 0; i < mass.size(); ++i) inverse_mass[i] = 1 / mass[i];
    inverse_trace_mass.resize(trace_mass.size());
    for (size_t i = 0; i < trace_mass.size(); ++i) inverse_trace_mass[i] = 1 / trace_mass[i];
    speeds.assign(face_count() * n, Speed{0, 0});
    Q = basis.points;
}
void Problem::interpolate(const double *nodal, double *pts) const {
    const Vec &V = basis.values;
    Vec t((size_t)Q * n);
    for (int v = 0; v < NVAR; ++v) {
        for (int iy = 0; iy < n; ++iy)  // t(qx, iy) = sum_ix V(qx, ix) U(ix, iy)
            for (int a = 0; a < Q; ++a) {
                double s = 0;
                for (int ix = 0; ix < n; ++ix) s += V[a * n + ix] * nodal[v * plane + ix + n * iy];
                t[a + Q * iy] = s;
            }
        for (int b = 0; b < Q; ++b)  // pts(qx, qy) = sum_iy t(qx, iy) V(qy, iy)
            for (int a = 0; a < Q; ++a) {
                double s = 0;
                for (int iy = 0; iy < n; ++iy) s += t[a + Q * iy] * V[b * n + iy];
                pts[v * Q * Q + a + Q * b] = s;
            }
    }
}
void Problem::subtract_weak_points(const double *fx, const double *fy, double *r) const {
    const double sx = .5 * hy, sy = .5 * hx;
    const Vec &V = basis.values, &wd = basis.wd, &qw = basis.qw;
    Vec t((size_t)n * Q);
    for (int v = 0; v < NVAR; ++v) {
        const double *x = fx + (size_t)v * Q * Q, *y = fy + (size_t)v * Q * Q;
        for (int b = 0; b < Q; ++b)  // t(i, qy) = sum_qx wd(qx, i) Fx(qx, qy)
            for (int i = 0; i < n; ++i) {
                double s = 0;
                for (int a = 0; a < Q; ++a) s += wd[a * n + i] * x[a + Q * b];
                t[i + n * b] = s;
            }
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double s = 0;
                for (int b = 0; b < Q; ++b) s += t[i + n * b] * qw[b] * V[b * n + j];
                r[v * plane + i + n * j] -= sx * s;
            }
        for (int b = 0; b < Q; ++b)  // t(i, qy) = sum_qx qw(qx) V(qx, i) Fy(qx, qy)
            for (int i = 0; i < n; ++i) {
                double s = 0;
                for (int a = 0; a < Q; ++a) s += qw[a] * V[a * n + i] * y[a + Q * b];
                t[i + n * b] = s;
            }
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double s = 0;
                for (int b = 0; b < Q; ++b) s += t[i + n * b] * wd[b * n + j];
                r[v * plane + i + n * j] -= sy * s;
            }
    }
}
int Problem::neighbor(int cell, int side) const {
    int x = cell % nx, y = cell / nx;
    if (side < 2) x = (x + (side == 0 ? nx - 1 : 1)) % nx;
    else y = (y + (side == 2 ? ny - 1 : 1)) % ny;
    return x + nx * y;
}
std::array<int, NFACES> Problem::faces(int cell) const {
    return {neighbor(cell, 0), cell, cells + neighbor(cell, 2), cells + cell};
}
double Problem::face_weight(int face, int q) const {
    return .5 * (face < cells ? hy : hx) * basis.w[q];
}
int Problem::face_node(int side, int q, int i) const { return side < 2 ? i + n * q : q + n * i; }
void Problem::face_values(const double *nodal, int side, double *values) const {
    const Vec &e = side % 2 ? basis.right : basis.left;
    for (int q = 0; q < n; ++q)
        for (int v = 0; v < NVAR; ++v) {
            double s = 0;
            for (int i = 0; i < n; ++i) s += e[i] * nodal[v * plane + face_node(side, q, i)];
            values[q * NVAR + v] = s;
        }
}
void Problem::lift(int side, const double *values, double *nodal, double scale) const {
    const Vec &e = side % 2 ? basis.right : basis.left;
    for (int q = 0; q < n; ++q)
        for (int v = 0; v < NVAR; ++v)
            for (int i = 0; i < n; ++i)
                nodal[v * plane + face_node(side, q, i)] += scale * e[i] * values[q * NVAR + v];
}
// tensor_product.cpp:41-56 (subtract_collocated): r -= (hy/2)(Dw)^T Fx W + (hx/2) W Fy Dw
void Problem::subtract_weak(const double *fx, const double *fy, double *r) const {
    const double sx = .5 * hy, sy = .5 * hx;
    const Vec &d = basis.dw, &w = basis.w;
    for (int v = 0; v < NVAR; ++v)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double wx = 0, wy = 0;
                for (int q = 0; q < n; ++q) {
                    wx += d[q * n + i] * fx[v * plane + q + n * j];
                    wy += fy[v * plane + i + n * q] * d[q * n + j];
                }
                r[v * plane + i + n * j] -= sx * w[j] * wx + sy * w[i] * wy;
            }
}
// discretization.cpp:111-122
void Problem::volume_residual(const Vec &u, Vec &r) const {
    r.resize(size());
    for (int i = 0; i < size(); ++i) r[i] = mass[i] * (u[i] - old[i]) / step_size;
    if (n == 1) return;
    if (Q != n) {
#pragma omp parallel
        {
            const int QQ = Q * Q;
            Vec pts((size_t)NVAR * QQ), fx((size_t)NVAR * QQ), fy((size_t)NVAR * QQ);
#pragma omp for schedule(static)
            for (int cell = 0; cell < cells; ++cell) {
                interpolate(u.data() + cell * block, pts.data());
                for (int q = 0; q < QQ; ++q) {
                    State s{pts[q], pts[QQ + q], pts[2 * QQ + q], pts[3 * QQ + q]};
                    State a = example.gas.flux(s, 0), b = example.gas.flux(s, 1);
                    for (int v = 0; v < NVAR; ++v) {
                        fx[v * QQ + q] = a[v];
                        fy[v * QQ + q] = b[v];
                    }
                }
                subtract_weak_points(fx.data(), fy.data(), r.data() + cell * block);
            }
        }
        return;
    }
#pragma omp parallel
    {
        Vec fx(block), fy(block);
#pragma omp for schedule(static)
        for (int cell = 0; cell < cells; ++cell) {
            const double *uc = u.data() + cell * block;
            for (int node = 0; node < plane; ++node) {
                State s{uc[node], uc[plane + node], uc[2 * plane + node], uc[3 * plane + node]};
                State a = example.gas.flux(s, 0), b = example.gas.flux(s, 1);
                for (int v = 0; v < NVAR; ++v) {
                    fx[v * plane + node] = a[v];
                    fy[v * plane + node] = b[v];
                }
            }
            subtract_weak(fx.data(), fy.data(), r.data() + cell * block);
        }
    }
}
// discretization.cpp:123-140 — each cell lifts its own two "left" faces (sides 1, 3) and the
// two faces it receives from its lower neighbours (sides 0, 2) so the loop is race-free.
void Problem::dg_residual(const Vec &u, Vec &r) const {
    volume_residual(u, r);
#pragma omp parallel
    {
        Vec l(n * NVAR), rr(n * NVAR), flux(n * NVAR);
#pragma omp for schedule(static)
        for (int cell = 0; cell < cells; ++cell) {
            for (int side = 0; side < NFACES; ++side) {
                const int axis = side / 2;
                const int lc = side % 2 ? cell : neighbor(cell, side);  // cell left of the face
                const int rc = neighbor(lc, 2 * axis + 1);
                const int face = axis * cells + lc;
                face_values(u.data() + lc * block, 2 * axis + 1, l.data());
                face_values(u.data() + rc * block, 2 * axis, rr.data());
                for (int q = 0; q < n; ++q) {
                    State L, R;
                    for (int v = 0; v < NVAR; ++v) { L[v] = l[q * NVAR + v]; R[v] = rr[q * NVAR + v]; }
                    const Speed s = speeds[face * n + q];
                    State fl = example.gas.flux(L, axis), fr = example.gas.flux(R, axis);
                    const double scale = face_weight(face, q) / (s.a + s.b);
                    for (int v = 0; v < NVAR; ++v)
                        flux[q * NVAR + v] = scale * (s.b * fl[v] + s.a * fr[v] + s.a * s.b * (L[v] - R[v]));
                }
                lift(side, flux.data(), r.data() + cell * block, side % 2 ? 1. : -1.);
            }
        }
    }
}
// discretization.cpp:141-162
void Problem::hybrid_residual(const Vec &u, const Vec &lambda, Vec &r, Vec &g) const {
    volume_residual(u, r);
    g.assign(trace_size(), 0.);
    Vec l(n * NVAR), rr(n * NVAR), ff(n * NVAR), of(n * NVAR);
    for (int axis = 0; axis < NDIM; ++axis)
        for (int cell = 0; cell < cells; ++cell) {
            const int side = 2 * axis + 1, next = neighbor(cell, side), face = axis * cells + cell;
            face_values(u.data() + cell * block, side, l.data());
            face_values(u.data() + next * block, side - 1, rr.data());
            for (int q = 0; q < n; ++q) {
                State L, R, z;
                for (int v = 0; v < NVAR; ++v) {
                    L[v] = l[q * NVAR + v];
                    R[v] = rr[q * NVAR + v];
                    z[v] = lambda[face * face_width() + v * n + q];
                }
                const Speed s = speeds[face * n + q];
                const double weight = face_weight(face, q);
                State fl = example.gas.flux(L, axis), fr = example.gas.flux(R, axis);
                for (int v = 0; v < NVAR; ++v) {
                    ff[q * NVAR + v] = weight * (fl[v] + s.a * (L[v] - z[v]));
                    of[q * NVAR + v] = weight * (fr[v] + s.b * (z[v] - R[v]));
                    g[face * face_width() + v * n + q] = ff[q * NVAR + v] - of[q * NVAR + v];
                }
            }
            lift(side, ff.data(), r.data() + cell * block);
            lift(side - 1, of.data(), r.data() + next * block, -1);
        }
}
// discretization.cpp:163-195
double Problem::freeze(const Vec &u) {
    old = u;
    Vec l(n * NVAR), rr(n * NVAR);
    for (int axis = 0; axis < NDIM; ++axis)
        for (int cell = 0; cell < cells; ++cell) {
            const int side = 2 * axis + 1, next = neighbor(cell, side), face = axis * cells + cell;
            face_values(u.data() + cell * block, side, l.data());
            face_values(u.data() + next * block, side - 1, rr.data());
            for (int q = 0; q < n; ++q) {
                State L, R;
                for (int v = 0; v < NVAR; ++v) { L[v] = l[q * NVAR + v]; R[v] = rr[q * NVAR + v]; }
                speeds[face * n + q] = einfeldt(L, R, example.gas, config.safety, axis);
            }
        }
    double rate = 0;
    for (int cell = 0; cell < cells; ++cell) {
        double alpha[2] = {0, 0};
        const auto fs = faces(cell);
        for (int side = 0; side < NFACES; ++side)
            for (int q = 0; q < n; ++q) {
                const Speed s = speeds[fs[side] * n + q];
                alpha[side / 2] = std::max({alpha[side / 2], s.a, s.b});
            }
        // discretization.cpp:184-192: the states at the volume points (the nodes when collocated)
        Vec pts;
        const double *uc = u.data() + cell * block;
        int npts = plane, stride = plane;
        if (Q != n) {
            pts.resize((size_t)NVAR * Q * Q);
            interpolate(uc, pts.data());
            uc = pts.data();
            npts = stride = Q * Q;
        }
        for (int node = 0; node < npts; ++node) {
            State s{uc[node], uc[stride + node], uc[2 * stride + node], uc[3 * stride + node]};
            double ir, vx, vy, p, H;
            example.gas.primitive(s, ir, vx, vy, p, H);
            require(s[Density] > 0 && p > 0, "Invalid CFL volume state");
            const double sound = std::sqrt(example.gas.gamma * p * ir);
            alpha[0] = std::max(alpha[0], std::abs(vx) + sound);
            alpha[1] = std::max(alpha[1], std::abs(vy) + sound);
        }
        rate = std::max(rate, alpha[0] / hx + alpha[1] / hy);
    }
    return rate;
}
// discretization.cpp:196-210
void Problem::trace(const Vec &u, Vec &lambda) const {
    lambda.assign(trace_size(), 0.);
    Vec l(n * NVAR), rr(n * NVAR);
    for (int axis = 0; axis < NDIM; ++axis)
        for (int cell = 0; cell < cells; ++cell) {
            const int side = 2 * axis + 1, next = neighbor(cell, side), face = axis * cells + cell;
            face_values(u.data() + cell * block, side, l.data());
            face_values(u.data() + next * block, side - 1, rr.data());
            for (int q = 0; q < n; ++q) {
                State L, R;
                for (int v = 0; v < NVAR; ++v) { L[v] = l[q * NVAR + v]; R[v] = rr[q * NVAR + v]; }
                const Speed s = speeds[face * n + q];
                State fl = example.gas.flux(L, axis), fr = example.gas.flux(R, axis);
                for (int v = 0; v < NVAR; ++v)
                    lambda[face * face_width() + v * n + q] =
                        (s.a * L[v] + s.b * R[v] + fl[v] - fr[v]) / (s.a + s.b);
            }
        }
}
// discretization.cpp:211-233
bool Problem::physical(const double *s, int count) const {
    for (int q = 0; q < count * NVAR; ++q)
        if (!std::isfinite(s[q])) return false;
    for (int q = 0; q < count; ++q) {
        State st{s[q * NVAR], s[q * NVAR + 1], s[q * NVAR + 2], s[q * NVAR + 3]};
        if (st[Density] <= 1e-13 || !(example.gas.pressure(st) > 1e-13)) return false;
    }
    return true;
}
bool Problem::admissible(const Vec &u) const {
    if ((int)u.size() != size()) return false;
    Vec pts(plane * NVAR), fv(n * NVAR);
    for (int cell = 0; cell < cells; ++cell) {
        const double *uc = u.data() + cell * block;
        for (int node = 0; node < plane; ++node)
            for (int v = 0; v < NVAR; ++v) pts[node * NVAR + v] = uc[v * plane + node];
        if (!physical(pts.data(), plane)) return false;
        if (Q != n) {  // discretization.cpp:224-227: also at the volume points
            Vec q((size_t)NVAR * Q * Q), qs((size_t)NVAR * Q * Q);
            interpolate(uc, q.data());
            for (int k = 0; k < Q * Q; ++k)
                for (int v = 0; v < NVAR; ++v) qs[k * NVAR + v] = q[v * Q * Q + k];
            if (!physical(qs.data(), Q * Q)) return false;
        }
        for (int side = 0; side < NFACES; ++side) {
            face_values(uc, side, fv.data());
            if (!physical(fv.data(), n)) return false;
        }
    }
    return true;
}
double Problem::residual_norm(const Vec &r) const {
    double s = 0;
    for (size_t i = 0; i < r.size(); ++i) s += r[i] * r[i] * inverse_mass[i];
    return std::sqrt(s / (example.lx * example.ly));
}
State Problem::integral(const Vec &u) const {
    State result{0, 0, 0, 0};
    for (int cell = 0; cell < cells; ++cell)
        for (int v = 0; v < NVAR; ++v)
            for (int node = 0; node < plane; ++node)
                result[v] += u[index(cell, v, node)] * mass[index(cell, v, node)];
    return result;
}
// initial_and_error.cpp:4-54 — L2 projection with a max(20,2n+3)-point rule, then a
// positivity scaling about the cell mean (collocated volume points coincide with nodes).
void Problem::initial(Vec &u) const {
    u.assign(size(), 0.);
    const int Q = (int)basis.ex.size();
    std::string failure;
#pragma omp parallel
    {
        Vec samples(Q * Q * NVAR), scratch(n * Q), checks;
#pragma omp for schedule(static)
        for (int cell = 0; cell < cells; ++cell) {
            try {
                for (int j = 0; j < Q; ++j)
                    for (int i = 0; i < Q; ++i) {
                        State e = example.exact(
                            -.5 * example.lx + hx * (cell % nx + .5) + .5 * hx * basis.ex[i],
                            -.5 * example.ly + hy * (cell / nx + .5) + .5 * hy * basis.ex[j], 0);
                        for (int v = 0; v < NVAR; ++v) samples[(i + Q * j) * NVAR + v] = e[v];
                    }
                double *uc = u.data() + cell * block;
                for (int v = 0; v < NVAR; ++v) {
                    // scratch(a, j) = sum_i P(a, i) S(i, j); U(a, b) = sum_j scratch(a, j) P(b, j)
                    for (int a = 0; a < n; ++a)
                        for (int j = 0; j < Q; ++j) {
                            double s = 0;
                            for (int i = 0; i < Q; ++i)
                                s += basis.projection[a * Q + i] * samples[(i + Q * j) * NVAR + v];
                            scratch[a * Q + j] = s;
                        }
                    for (int a = 0; a < n; ++a)
                        for (int b = 0; b < n; ++b) {
                            double s = 0;
                            for (int j = 0; j < Q; ++j) s += scratch[a * Q + j] * basis.projection[b * Q + j];
                            uc[v * plane + a + n * b] = s;
                        }
                }
                State mean{0, 0, 0, 0};
                for (int j = 0; j < n; ++j)
                    for (int i = 0; i < n; ++i)
                        for (int v = 0; v < NVAR; ++v)
                            mean[v] += .25 * basis.w[i] * basis.w[j] * uc[v * plane + i + n * j];
                require(mean[Density] > 0 && example.gas.pressure(mean) > 0, "Nonphysical cell average");
                // check points: nodes, volume points (= nodes), error-rule points, face points
                checks.clear();
                for (int rep = 0; rep < 2; ++rep)
                    for (int node = 0; node < plane; ++node)
                        for (int v = 0; v < NVAR; ++v) checks.push_back(uc[v * plane + node]);
                for (int j = 0; j < Q; ++j)
                    for (int i = 0; i < Q; ++i)
                        for (int v = 0; v < NVAR; ++v) {
                            double s = 0;
                            for (int b = 0; b < n; ++b)
                                for (int a = 0; a < n; ++a)
                                    s += basis.evalues[i * n + a] * basis.evalues[j * n + b] * uc[v * plane + a + n * b];
                            checks.push_back(s);
                        }
                Vec fv(n * NVAR);
                for (int side = 0; side < NFACES; ++side) {
                    face_values(uc, side, fv.data());
                    checks.insert(checks.end(), fv.begin(), fv.end());
                }
                double theta = 1;
                const int count = (int)checks.size() / NVAR;
                for (int q = 0; q < count; ++q) {
                    State diff;
                    for (int v = 0; v < NVAR; ++v) diff[v] = checks[q * NVAR + v] - mean[v];
                    auto phys = [&](double factor) {
                        State z;
                        for (int v = 0; v < NVAR; ++v) z[v] = mean[v] + factor * diff[v];
                        return z[Density] > 1e-12 && example.gas.pressure(z) > 1e-12;
                    };
                    if (!phys(theta)) {
                        double low = 0, high = theta;
                        for (int it = 0; it < 60; ++it) {
                            double middle = .5 * (low + high);
                            if (phys(middle)) low = middle; else high = middle;
                        }
                        theta = .99 * low;
                    }
                }
                for (int v = 0; v < NVAR; ++v)
                    for (int node = 0; node < plane; ++node)
                        uc[v * plane + node] = mean[v] + theta * (uc[v * plane + node] - mean[v]);
            } catch (const std::exception &e) {
#pragma omp critical
                failure = e.what();
            }
        }
    }
    require(failure.empty(), failure.c_str());
    require(admissible(u), "Invalid projected initial state");
}
// initial_and_error.cpp:55-73
State Problem::error(const Vec &u, double time) const {
    const int Q = (int)basis.ex.size();
    State result{0, 0, 0, 0};
    std::vector<State> partial(cells);
#pragma omp parallel for schedule(static)
    for (int cell = 0; cell < cells; ++cell) {
        State acc{0, 0, 0, 0};
        const double *uc = u.data() + cell * block;
        for (int j = 0; j < Q; ++j)
            for (int i = 0; i < Q; ++i) {
                State val{0, 0, 0, 0};
                for (int v = 0; v < NVAR; ++v)
                    for (int b = 0; b < n; ++b)
                        for (int a = 0; a < n; ++a)
                            val[v] += basis.evalues[i * n + a] * basis.evalues[j * n + b] * uc[v * plane + a + n * b];
                State e = example.exact(-.5 * example.lx + hx * (cell % nx + .5) + .5 * hx * basis.ex[i],
                                        -.5 * example.ly + hy * (cell / nx + .5) + .5 * hy * basis.ex[j], time);
                for (int v = 0; v < NVAR; ++v) {
                    const double d = val[v] - e[v];
                    acc[v] += .25 * hx * hy * basis.ew[i] * basis.ew[j] * d * d;
                }
            }
        partial[cell] = acc;
    }
    for (int cell = 0; cell < cells; ++cell)
        for (int v = 0; v < NVAR; ++v) result[v] += partial[cell][v];
    for (int v = 0; v < NVAR; ++v) result[v] = std::sqrt(result[v]);
    return result;
}

// ---------------------------------------------------------------- volume/face jacobian, DG operator
DGOperator::DGOperator(const Problem &p) : p_(p) {
    const int nf = p.face_count(), n = p.n;
    prim_.assign((size_t)p.cells * p.Q * p.Q * 3, 0.);
    fl_.assign((size_t)nf * n * 3, 0.);
    fr_.assign((size_t)nf * n * 3, 0.);
    tau_l_.assign(nf * n, 0.); tau_r_ = tau_l_; blend_l_ = tau_l_; blend_r_ = tau_l_; penalty_ = tau_l_;
    weights_.assign(nf * n, 0.);
    for (int f = 0; f < nf; ++f)
        for (int q = 0; q < n; ++q) weights_[f * n + q] = p.face_weight(f, q);
    diagonal_.assign(p.trace_size(), 0.);
}
// volume_jacobian.cpp:30-42 and face_jacobian.cpp:16-37
void DGOperator::refresh(const Vec &u) {
    const Problem &p = p_;
    require(p.step_size > 0, "Set the time step before refreshing the Jacobian");
    inverse_step_ = 1 / p.step_size;
    const int n = p.n, plane = p.plane;
    if (n > 1 && p.Q != n) {  // volume_jacobian.cpp:33-38: primitives at the volume points
        const int QQ = p.Q * p.Q;
        Vec pts((size_t)NVAR * QQ);
        for (int cell = 0; cell < p.cells; ++cell) {
            p.interpolate(u.data() + cell * p.block, pts.data());
            for (int q = 0; q < QQ; ++q) {
                State s{pts[q], pts[QQ + q], pts[2 * QQ + q], pts[3 * QQ + q]};
                double ir, vx, vy, pr, H;
                p.example.gas.primitive(s, ir, vx, vy, pr, H);
                double *c = &prim_[((size_t)cell * QQ + q) * 3];
                c[0] = vx; c[1] = vy; c[2] = H;
            }
        }
    } else if (n > 1)
        for (int cell = 0; cell < p.cells; ++cell)
            for (int node = 0; node < plane; ++node) {
                const double *uc = u.data() + cell * p.block;
                State s{uc[node], uc[plane + node], uc[2 * plane + node], uc[3 * plane + node]};
                double ir, vx, vy, pr, H;
                p.example.gas.primitive(s, ir, vx, vy, pr, H);
                double *c = &prim_[((size_t)cell * plane + node) * 3];
                c[0] = vx; c[1] = vy; c[2] = H;
            }
    Vec l(n * NVAR), r(n * NVAR);
    for (int axis = 0; axis < NDIM; ++axis)
        for (int cell = 0; cell < p.cells; ++cell) {
            const int face = axis * p.cells + cell, side = 2 * axis + 1;
            p.face_values(u.data() + cell * p.block, side, l.data());
            p.face_values(u.data() + p.neighbor(cell, side) * p.block, side - 1, r.data());
            for (int q = 0; q < n; ++q) {
                State L, R;
                for (int v = 0; v < NVAR; ++v) { L[v] = l[q * NVAR + v]; R[v] = r[q * NVAR + v]; }
                double ir, vx, vy, pr, H;
                p.example.gas.primitive(L, ir, vx, vy, pr, H);
                double *cl = &fl_[((size_t)face * n + q) * 3];
                cl[0] = vx; cl[1] = vy; cl[2] = H;
                p.example.gas.primitive(R, ir, vx, vy, pr, H);
                double *cr = &fr_[((size_t)face * n + q) * 3];
                cr[0] = vx; cr[1] = vy; cr[2] = H;
                const Speed s = p.speeds[face * n + q];
                const double w = weights_[face * n + q];
                tau_l_[face * n + q] = s.a;
                tau_r_[face * n + q] = s.b;
                blend_l_[face * n + q] = w * s.b / (s.a + s.b);
                blend_r_[face * n + q] = w * s.a / (s.a + s.b);
                penalty_[face * n + q] = w * s.a * s.b / (s.a + s.b);
                for (int v = 0; v < NVAR; ++v)
                    diagonal_[face * p.face_width() + v * n + q] = -w * (s.a + s.b);
            }
        }
    ready_ = true;
}
// volume_jacobian.cpp:43-58 / face_jacobian.cpp:38-55: linearised flux from (u,v,H)
void DGOperator::normal_action(const double *c, const double *d, double *out, int axis) const {
    const double u = c[0], v = c[1], H = c[2];
    const double dr = d[0], dx = d[1], dy = d[2], de = d[3];
    const double dp = (p_.example.gas.gamma - 1.) * (de - u * dx - v * dy + .5 * (u * u + v * v) * dr);
    if (axis == 0) {
        out[0] = dx;
        out[1] = 2 * u * dx - u * u * dr + dp;
        out[2] = u * dy + v * dx - u * v * dr;
        out[3] = H * (dx - u * dr) + u * (de + dp);
    } else {
        out[0] = dy;
        out[1] = u * dy + v * dx - u * v * dr;
        out[2] = 2 * v * dy - v * v * dr + dp;
        out[3] = H * (dy - v * dr) + v * (de + dp);
    }
}
// volume_jacobian.cpp:59-71 + dg_operator.cpp:10-21
void DGOperator::apply(const Vec &d, Vec &out) const {
    const Problem &p = p_;
    require(ready_, "Refresh the volume Jacobian before applying it");
    out.resize(p.size());
    for (int i = 0; i < p.size(); ++i) out[i] = p.mass[i] * d[i] * inverse_step_;
    const int n = p.n, plane = p.plane, blk = p.block;
#pragma omp parallel
    {
        Vec fx(blk), fy(blk), l(n * NVAR), r(n * NVAR), flux(n * NVAR);
#pragma omp for schedule(static)
        for (int cell = 0; cell < p.cells; ++cell) {
            double *oc = out.data() + cell * blk;
            if (n > 1 && p.Q != n) {  // volume_jacobian.cpp:64-69: the direction at the points
                const int QQ = p.Q * p.Q;
                Vec pd((size_t)NVAR * QQ), px((size_t)NVAR * QQ), py((size_t)NVAR * QQ);
                p.interpolate(d.data() + cell * blk, pd.data());
                for (int q = 0; q < QQ; ++q) {
                    double dd[4] = {pd[q], pd[QQ + q], pd[2 * QQ + q], pd[3 * QQ + q]};
                    double ax[4], ay[4];
                    const double *c = &prim_[((size_t)cell * QQ + q) * 3];
                    normal_action(c, dd, ax, 0);
                    normal_action(c, dd, ay, 1);
                    for (int v = 0; v < NVAR; ++v) { px[v * QQ + q] = ax[v]; py[v * QQ + q] = ay[v]; }
                }
                p.subtract_weak_points(px.data(), py.data(), oc);
            } else if (n > 1) {
                const double *dc = d.data() + cell * blk;
                for (int node = 0; node < plane; ++node) {
                    double dd[4] = {dc[node], dc[plane + node], dc[2 * plane + node], dc[3 * plane + node]};
                    double ax[4], ay[4];
                    const double *c = &prim_[((size_t)cell * plane + node) * 3];
                    normal_action(c, dd, ax, 0);
                    normal_action(c, dd, ay, 1);
                    for (int v = 0; v < NVAR; ++v) { fx[v * plane + node] = ax[v]; fy[v * plane + node] = ay[v]; }
                }
                const double sx = .5 * p.hy, sy = .5 * p.hx;
                const Vec &dw = p.basis.dw, &w = p.basis.w;
                for (int v = 0; v < NVAR; ++v)
                    for (int j = 0; j < n; ++j)
                        for (int i = 0; i < n; ++i) {
                            double wx = 0, wy = 0;
                            for (int q = 0; q < n; ++q) {
                                wx += dw[q * n + i] * fx[v * plane + q + n * j];
                                wy += fy[v * plane + i + n * q] * dw[q * n + j];
                            }
                            oc[v * plane + i + n * j] -= sx * w[j] * wx + sy * w[i] * wy;
                        }
            }
            for (int side = 0; side < NFACES; ++side) {
                const int axis = side / 2;
                const int lc = side % 2 ? cell : p.neighbor(cell, side);
                const int rc = p.neighbor(lc, 2 * axis + 1);
                const int face = axis * p.cells + lc;
                p.face_values(d.data() + lc * blk, 2 * axis + 1, l.data());
                p.face_values(d.data() + rc * blk, 2 * axis, r.data());
                for (int q = 0; q < n; ++q) {
                    double al[4], ar[4];
                    normal_action(&fl_[((size_t)face * n + q) * 3], &l[q * NVAR], al, axis);
                    normal_action(&fr_[((size_t)face * n + q) * 3], &r[q * NVAR], ar, axis);
                    const int k = face * n + q;
                    for (int v = 0; v < NVAR; ++v)
                        flux[q * NVAR + v] = blend_l_[k] * al[v] + blend_r_[k] * ar[v] +
                                             penalty_[k] * (l[q * NVAR + v] - r[q * NVAR + v]);
                }
                p.lift(side, flux.data(), oc, side % 2 ? 1. : -1.);
            }
        }
    }
}
// face_jacobian.cpp:65-82
Jac DGOperator::physical(int face, int q, bool left) const {
    const double *c = left ? &fl_[((size_t)face * p_.n + q) * 3] : &fr_[((size_t)face * p_.n + q) * 3];
    return p_.example.gas.cached_jacobian(c[0], c[1], c[2], face / p_.cells);
}
Jac DGOperator::hll(int face, int q, bool left) const {
    Jac a = physical(face, q, left);
    const int k = face * p_.n + q;
    const double b = left ? blend_l_[k] : blend_r_[k];
    for (double &x : a) x *= b;
    for (int v = 0; v < NVAR; ++v) a[v * 4 + v] += left ? penalty_[k] : -penalty_[k];
    return a;
}
double DGOperator::tau(int face, int q, bool left) const {
    return left ? tau_l_[face * p_.n + q] : tau_r_[face * p_.n + q];
}
Jac DGOperator::hdg(int face, int q, bool left) const {
    Jac a = physical(face, q, left);
    const double sign = left ? 1. : -1.;
    for (double &x : a) x *= sign;
    for (int v = 0; v < NVAR; ++v) a[v * 4 + v] += tau(face, q, left);
    const double w = weights_[face * p_.n + q];
    for (double &x : a) x *= w;
    return a;
}
// volume_jacobian.cpp:72-89,117-126 (collocated block, mass/tau on the diagonal)
void DGOperator::volume_block(int cell, double *out) const {
    const Problem &p = p_;
    require(ready_, "Refresh the volume Jacobian before assembling a block");
    const int n = p.n, plane = p.plane, m = p.block;
    std::fill(out, out + (size_t)m * m, 0.);
    if (n > 1 && p.Q != n) {
        // volume_jacobian.cpp:90-116: d r(v, i, j) / d U(w, k, l) summed over the points (a, b):
        // -(hy/2) wd(a,i) X(v,w) V(a,k) V(b,l) qw(b) V(b,j) - (hx/2) qw(a) V(a,i) Y(v,w) V(a,k) V(b,l) wd(b,j)
        const int Q = p.Q;
        const Vec &V = p.basis.values, &wd = p.basis.wd, &qw = p.basis.qw;
        std::vector<Jac> X((size_t)Q * Q), Y((size_t)Q * Q);
        for (int q = 0; q < Q * Q; ++q) {
            const double *c = &prim_[((size_t)cell * Q * Q + q) * 3];
            X[q] = p.example.gas.cached_jacobian(c[0], c[1], c[2], 0);
            Y[q] = p.example.gas.cached_jacobian(c[0], c[1], c[2], 1);
        }
        Vec lx((size_t)n * n), ly((size_t)n * n);  // [k][i] for one (b, v, w)
        for (int b = 0; b < Q; ++b)
            for (int wv = 0; wv < NVAR; ++wv)
                for (int v = 0; v < NVAR; ++v) {
                    for (int k = 0; k < n; ++k)
                        for (int i = 0; i < n; ++i) {
                            double sxv = 0, syv = 0;
                            for (int a = 0; a < Q; ++a) {
                                const int q = a + Q * b;
                                sxv += wd[a * n + i] * X[q][v * 4 + wv] * V[a * n + k];
                                syv += qw[a] * V[a * n + i] * Y[q][v * 4 + wv] * V[a * n + k];
                            }
                            lx[k * n + i] = -sxv;
                            ly[k * n + i] = -syv;
                        }
                    for (int l = 0; l < n; ++l)
                        for (int k = 0; k < n; ++k) {
                            double *column = out + (size_t)p.local(wv, k + n * l) * m;
                            for (int j = 0; j < n; ++j) {
                                const double cx = .5 * p.hy * qw[b] * V[b * n + j] * V[b * n + l];
                                const double cy = .5 * p.hx * wd[b * n + j] * V[b * n + l];
                                for (int i = 0; i < n; ++i)
                                    column[v * plane + n * j + i] += cx * lx[k * n + i] + cy * ly[k * n + i];
                            }
                        }
                }
    } else if (n > 1) {
        const Vec &dw = p.basis.dw, &w = p.basis.w;
        for (int jy = 0; jy < n; ++jy)
            for (int jx = 0; jx < n; ++jx) {
                const int node = jx + n * jy;
                const double *c = &prim_[((size_t)cell * plane + node) * 3];
                const Jac X = p.example.gas.cached_jacobian(c[0], c[1], c[2], 0);
                const Jac Y = p.example.gas.cached_jacobian(c[0], c[1], c[2], 1);
                for (int wv = 0; wv < NVAR; ++wv) {
                    double *column = out + (size_t)p.local(wv, node) * m;
                    for (int v = 0; v < NVAR; ++v) {
                        const double sx = .5 * p.hy * w[jy] * X[v * 4 + wv];
                        for (int i = 0; i < n; ++i) column[v * plane + n * jy + i] -= sx * dw[jx * n + i];
                        const double sy = -.5 * p.hx * w[jx] * Y[v * 4 + wv];
                        for (int iy = 0; iy < n; ++iy) column[v * plane + jx + n * iy] += sy * dw[jy * n + iy];
                    }
                }
            }
    }
    for (int i = 0; i < m; ++i) out[(size_t)i * m + i] += p.mass[(size_t)cell * m + i] * inverse_step_;
}
// dg_operator.cpp:22-48
void DGOperator::block(int row, int col, double *out) const {
    const Problem &p = p_;
    const int m = p.block, n = p.n;
    if (row == col) volume_block(row, out);
    else std::fill(out, out + (size_t)m * m, 0.);
    const auto fs = p.faces(row);
    for (int side = 0; side < NFACES; ++side) {
        if (col != row && col != p.neighbor(row, side)) continue;
        const bool left = col == (fs[side] % p.cells);
        const int trial_side = 2 * (side / 2) + (left ? 1 : 0);
        const Vec &test = side % 2 ? p.basis.right : p.basis.left;
        const Vec &trial = left ? p.basis.right : p.basis.left;
        const double sign = side % 2 ? 1 : -1;
        for (int q = 0; q < n; ++q) {
            const Jac der = hll(fs[side], q, left);
            for (int wv = 0; wv < NVAR; ++wv)
                for (int j = 0; j < n; ++j) {
                    double *column = out + (size_t)p.local(wv, p.face_node(trial_side, q, j)) * m;
                    for (int v = 0; v < NVAR; ++v) {
                        const double scale = sign * trial[j] * der[v * 4 + wv];
                        for (int i = 0; i < n; ++i) column[p.local(v, p.face_node(side, q, i))] += scale * test[i];
                    }
                }
        }
    }
}
// J^T w assembled from the five coupling blocks of each block row (dense, small meshes only).
void DGOperator::apply_transpose(const Vec &wv, Vec &out) const {
    const Problem &p = p_;
    const int m = p.block;
    out.assign(p.size(), 0.);
    Vec blk((size_t)m * m);
    for (int row = 0; row < p.cells; ++row) {
        int cols[5] = {row, p.neighbor(row, 0), p.neighbor(row, 1), p.neighbor(row, 2), p.neighbor(row, 3)};
        for (int k = 0; k < 5; ++k) {
            block(row, cols[k], blk.data());
            for (int c = 0; c < m; ++c) {
                double s = 0;
                for (int r = 0; r < m; ++r) s += blk[(size_t)c * m + r] * wv[(size_t)row * m + r];
                out[(size_t)cols[k] * m + c] += s;
            }
        }
    }
}

// ---------------------------------------------------------------- dense LU (row partial pivoting)
void DenseLU::compute(const double *a, int width) {
    m = width;
    lu.assign(a, a + (size_t)m * m);
    for (size_t i = 0; i < lu.size(); ++i) require(std::isfinite(lu[i]), "Nonfinite block LU input");
    perm.resize(m);
    for (int i = 0; i < m; ++i) perm[i] = i;
    for (int k = 0; k < m; ++k) {
        int piv = k;
        double best = std::abs(lu[(size_t)k * m + k]);
        for (int i = k + 1; i < m; ++i) {
            const double v = std::abs(lu[(size_t)k * m + i]);
            if (v > best) { best = v; piv = i; }
        }
        if (piv != k) {
            for (int j = 0; j < m; ++j) std::swap(lu[(size_t)j * m + k], lu[(size_t)j * m + piv]);
            std::swap(perm[k], perm[piv]);
        }
        const double pivot = lu[(size_t)k * m + k];
        if (pivot != 0)
            for (int i = k + 1; i < m; ++i) lu[(size_t)k * m + i] /= pivot;
        for (int j = k + 1; j < m; ++j) {
            const double ukj = lu[(size_t)j * m + k];
            if (ukj == 0) continue;
            double *cj = &lu[(size_t)j * m];
            const double *ck = &lu[(size_t)k * m];
            for (int i = k + 1; i < m; ++i) cj[i] -= ck[i] * ukj;
        }
    }
    for (int i = 0; i < m; ++i)
        require(std::isfinite(lu[(size_t)i * m + i]) &&
                    std::abs(lu[(size_t)i * m + i]) > std::numeric_limits<double>::min(),
                "Singular or nonfinite LU factors");
    for (size_t i = 0; i < lu.size(); ++i) require(std::isfinite(lu[i]), "Singular or nonfinite LU factors");
}
void DenseLU::solve(const double *b, double *x) const {
    Vec t(m);
    for (int i = 0; i < m; ++i) t[i] = b[perm[i]];
    for (int j = 0; j < m; ++j) {
        const double tj = t[j];
        if (tj != 0)
            for (int i = j + 1; i < m; ++i) t[i] -= lu[(size_t)j * m + i] * tj;
    }
    for (int j = m - 1; j >= 0; --j) {
        t[j] /= lu[(size_t)j * m + j];
        const double tj = t[j];
        if (tj != 0)
            for (int i = 0; i < j; ++i) t[i] -= lu[(size_t)j * m + i] * tj;
    }
    for (int i = 0; i < m; ++i) x[i] = t[i];
}
// dense_lu.hpp:42-49: row by row, solve with U^T (lower, U's diagonal), then L^T (unit upper),
// then apply P^T.
void DenseLU::right_solve(double *x) const {
    Vec s(m);
    for (int r = 0; r < m; ++r) {
        for (int i = 0; i < m; ++i) s[i] = x[(size_t)i * m + r];
        for (int i = 0; i < m; ++i) {
            double v = s[i];
            for (int k = 0; k < i; ++k) v -= lu[(size_t)i * m + k] * s[k];  // U(k, i) = lu[i*m + k]
            s[i] = v / lu[(size_t)i * m + i];
        }
        for (int i = m - 1; i >= 0; --i) {
            double v = s[i];
            for (int k = i + 1; k < m; ++k) v -= lu[(size_t)i * m + k] * s[k];  // L(k, i) = lu[i*m + k]
            s[i] = v;
        }
        for (int i = 0; i < m; ++i) x[(size_t)perm[i] * m + r] = s[i];
    }
}
std::vector<std::vector<int>> periodic_adjacency(int cells) {
    std::vector<std::vector<int>> adj(cells);
    for (int c = 0; c < cells; ++c) adj[c] = {(c + cells - 1) % cells, c, (c + 1) % cells};
    return adj;
}
std::vector<std::vector<int>> cartesian_adjacency(int nx, int ny) {
    std::vector<std::vector<int>> adj((size_t)nx * ny);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x)
            adj[x + nx * y] = {x + nx * y, (x + nx - 1) % nx + nx * y, (x + 1) % nx + nx * y, x + nx * ((y + ny - 1) % ny),
                               x + nx * ((y + 1) % ny)};
    return adj;
}
BlockILU0::BlockILU0(const std::vector<std::vector<int>> &adjacency, int w)
    : rows((int)adjacency.size()), width(w), row_ptr(rows + 1, 0), diag(rows), lus(rows) {
    for (int r = 0; r < rows; ++r) {
        auto row = adjacency[r];
        row.push_back(r);
        std::sort(row.begin(), row.end());
        row.erase(std::unique(row.begin(), row.end()), row.end());
        col_idx.insert(col_idx.end(), row.begin(), row.end());
        row_ptr[r + 1] = (int)col_idx.size();
    }
    values.assign(col_idx.size() * (size_t)w * w, 0.);
    upd_off.assign(col_idx.size() + 1, 0);
    for (int row = 0; row < rows; ++row) {
        diag[row] = find(row, row);
        for (int slot = row_ptr[row]; slot < row_ptr[row + 1]; ++slot) {
            upd_off[slot] = (int)upd_target.size();
            const int elim = col_idx[slot];
            if (elim >= row) continue;
            for (int upper = row_ptr[elim]; upper < row_ptr[elim + 1]; ++upper) {
                const int column = col_idx[upper];
                if (column <= elim) continue;
                const int target = find(row, column);
                if (target >= 0) {
                    upd_target.push_back(target);
                    upd_upper.push_back(upper);
                }
            }
        }
    }
    upd_off.back() = (int)upd_target.size();
}
int BlockILU0::find(int row, int col) const {
    for (int p = row_ptr[row]; p < row_ptr[row + 1]; ++p)
        if (col_idx[p] == col) return p;
    return -1;
}
// block_ilu.cpp:48-61 (factorize) after the provider filled every pattern block.
void BlockILU0::refresh(const std::function<void(int, int, double *)> &provider) {
    for (int row = 0; row < rows; ++row)
        for (int p = row_ptr[row]; p < row_ptr[row + 1]; ++p) provider(row, col_idx[p], block(p));
    const int w = width;
    for (int i = 0; i < rows; ++i) {
        for (int p = row_ptr[i]; p < diag[i]; ++p) {
            lus[col_idx[p]].right_solve(block(p));
            for (int u = upd_off[p]; u < upd_off[p + 1]; ++u) {
                // dense_lu.hpp:53-57: destination.col(j) -= right(k, j) * left.col(k)
                double *dst = block(upd_target[u]);
                const double *left = block(p), *right = block(upd_upper[u]);
                for (int j = 0; j < w; ++j)
                    for (int k = 0; k < w; ++k) {
                        const double r = right[(size_t)j * w + k];
                        for (int q = 0; q < w; ++q) dst[(size_t)j * w + q] -= r * left[(size_t)k * w + q];
                    }
            }
        }
        lus[i].compute(block(diag[i]), w);
    }
}
// block_ilu.cpp:62-84 (apply, natural order)
void BlockILU0::apply(const Vec &rhs, Vec &result) const {
    const int w = width;
    Vec work(rhs.begin(), rhs.end());
    auto gemv_sub = [&](const double *blk, int row, int col) {
        for (int k = 0; k < w; ++k) {
            const double xk = work[(size_t)col * w + k];
            for (int q = 0; q < w; ++q) work[(size_t)row * w + q] -= blk[(size_t)k * w + q] * xk;
        }
    };
    for (int i = 0; i < rows; ++i)
        for (int p = row_ptr[i]; p < diag[i]; ++p) gemv_sub(block(p), i, col_idx[p]);
    for (int i = rows - 1; i >= 0; --i) {
        for (int p = diag[i] + 1; p < row_ptr[i + 1]; ++p) gemv_sub(block(p), i, col_idx[p]);
        lus[i].solve(&work[(size_t)i * w], &work[(size_t)i * w]);
    }
    result = work;
}
BlockJacobi::BlockJacobi(int b, int w) : blocks(b), width(w), lus(b) {}
void BlockJacobi::refresh(const std::function<void(int, int, double *)> &provider) {
    std::string failure;
#pragma omp parallel
    {
        Vec blk((size_t)width * width);
#pragma omp for schedule(dynamic, 4)
        for (int i = 0; i < blocks; ++i) {
            provider(i, i, blk.data());
            try {
                lus[i].compute(blk.data(), width);
            } catch (const std::exception &) {
#pragma omp critical
                failure = "Singular block Jacobi factor";
            }
        }
    }
    require(failure.empty(), "Singular block Jacobi factor");
}
void BlockJacobi::apply(const Vec &rhs, Vec &result) const {
    result.resize(rhs.size());
#pragma omp parallel for schedule(static)
    for (int i = 0; i < blocks; ++i) lus[i].solve(rhs.data() + (size_t)i * width, result.data() + (size_t)i * width);
}

// ---------------------------------------------------------------- gmres.cpp:17-86
GMRES::GMRES(int n, int restart, const Vec &weights)
    : n_(n), restart_(std::min(n, restart)), basis_(restart_ + 1, Vec(n)),
      h_((size_t)(restart_ + 1) * restart_), cosine_(restart_), sine_(restart_), g_(restart_ + 1),
      y_(restart_), work_(n), residual_(n), column_(n), weights_(weights), proj_(restart_ + 1) {
    bool ok = n > 0 && restart > 0 && (int)weights_.size() == n;
    for (double w : weights_) ok = ok && std::isfinite(w) && w > 0;
    require(ok, "Invalid GMRES metric or dimensions");
}
double GMRES::dot(const Vec &a, const Vec &b) const {
    double s = 0;
    for (int i = 0; i < n_; ++i) s += a[i] * weights_[i] * b[i];
    return s;
}
double GMRES::norm(const Vec &a) const { return std::sqrt(std::max(0.0, dot(a, a))); }
LinearResult GMRES::solve(Action A, Action M, const Vec &rhs, Vec &x, int limit, double tolerance) {
    auto H = [&](int i, int j) -> double & { return h_[(size_t)j * (restart_ + 1) + i]; };
    x.assign(n_, 0.);
    residual_ = rhs;
    const double rhs_norm = norm(rhs);
    if (rhs_norm == 0) return {0, 0};
    int iterations = 0;
    while (iterations < limit) {
        const double beta = norm(residual_);
        if (beta <= tolerance * rhs_norm) return {iterations, beta / rhs_norm};
        for (int i = 0; i < n_; ++i) basis_[0][i] = residual_[i] / beta;
        std::fill(h_.begin(), h_.end(), 0.);
        std::fill(g_.begin(), g_.end(), 0.);
        g_[0] = beta;
        int count = 0;
        for (int j = 0; j < restart_ && iterations < limit; ++j) {
            column_ = basis_[j];
            M(column_, work_);
            A(work_, column_);
            for (int pass = 0; pass < 2; ++pass) {
                for (int k = 0; k <= j; ++k) {
                    double s = 0;
                    const Vec &b = basis_[k];
                    for (int i = 0; i < n_; ++i) s += b[i] * (weights_[i] * column_[i]);
                    proj_[k] = s;
                    H(k, j) += s;
                }
                for (int i = 0; i < n_; ++i) {
                    double s = 0;
                    for (int k = 0; k <= j; ++k) s += basis_[k][i] * proj_[k];
                    column_[i] -= s;
                }
            }
            const double next = norm(column_);
            H(j + 1, j) = next;
            if (next > 0)
                for (int i = 0; i < n_; ++i) basis_[j + 1][i] = column_[i] / next;
            for (int i = 0; i < j; ++i) {
                const double a = H(i, j), b = H(i + 1, j);
                H(i, j) = cosine_[i] * a + sine_[i] * b;
                H(i + 1, j) = -sine_[i] * a + cosine_[i] * b;
            }
            const double d = std::hypot(H(j, j), H(j + 1, j));
            require(std::isfinite(d) && d > 0, "GMRES Arnoldi breakdown");
            cosine_[j] = H(j, j) / d;
            sine_[j] = H(j + 1, j) / d;
            H(j, j) = d;
            H(j + 1, j) = 0;
            g_[j + 1] = -sine_[j] * g_[j];
            g_[j] *= cosine_[j];
            ++iterations;
            count = j + 1;
            if (std::abs(g_[j + 1]) <= tolerance * rhs_norm || next <= std::numeric_limits<double>::min())
                break;
        }
        for (int i = count - 1; i >= 0; --i) {
            double value = g_[i];
            for (int j = i + 1; j < count; ++j) value -= H(i, j) * y_[j];
            y_[i] = value / H(i, i);
        }
        for (int i = 0; i < n_; ++i) {
            double s = 0;
            for (int k = 0; k < count; ++k) s += basis_[k][i] * y_[k];
            work_[i] = s;
        }
        M(work_, column_);
        for (int i = 0; i < n_; ++i) x[i] += column_[i];
        A(x, work_);
        for (int i = 0; i < n_; ++i) residual_[i] = rhs[i] - work_[i];
        const double relative = norm(residual_) / rhs_norm;
        require(std::isfinite(relative), "Nonfinite GMRES residual");
        if (relative <= tolerance) return {iterations, relative};
    }
    throw std::runtime_error("GMRES iteration limit reached");
}

// ---------------------------------------------------------------- hybrid.cpp
HybridOperator::HybridOperator(const Problem &p) : p_(p), lin_(p) {
    const size_t m = p.block, t = p.local_trace_size();
    x_.assign(m * t * p.cells, 0.);
    schur_.assign(t * t * p.cells, 0.);
    y_.assign(m * p.cells, 0.);
    rhs_.assign(p.trace_size(), 0.);
}
// hybrid.cpp:28-30,56-72 with assemble_cell (31-55) and cell_c_many (face_jacobian.cpp:88-110)
void HybridOperator::refresh_projected(const Vec &u, const Vec &r) {
    const Problem &p = p_;
    lin_.refresh(u);
    std::fill(rhs_.begin(), rhs_.end(), 0.);  // skeleton residual g = 0 on the projected trace
    const int m = p.block, t = p.local_trace_size(), n = p.n, fw = p.face_width();
    Vec cy_all((size_t)t * p.cells);
    std::string failure;
#pragma omp parallel
    {
        Vec a((size_t)m * m), rhs((size_t)m * (t + 1)), solved((size_t)m * (t + 1)), act((size_t)t * (t + 1));
        Vec samples((size_t)n * NVAR);
        DenseLU lu;
#pragma omp for schedule(dynamic, 2)
        for (int cell = 0; cell < p.cells; ++cell) {
            lin_.volume_block(cell, a.data());
            std::fill(rhs.begin(), rhs.end(), 0.);
            const auto fs = p.faces(cell);
            for (int side = 0; side < NFACES; ++side) {
                const Vec &shape = side % 2 ? p.basis.right : p.basis.left;
                const bool left = side % 2 != 0;
                for (int q = 0; q < n; ++q) {
                    const Jac der = lin_.hdg(fs[side], q, left);
                    const double stab = p.face_weight(fs[side], q) * lin_.tau(fs[side], q, left);
                    for (int v = 0; v < NVAR; ++v)
                        for (int i = 0; i < n; ++i)
                            rhs[(size_t)(side * fw + v * n + q) * m + p.local(v, p.face_node(side, q, i))] =
                                -stab * shape[i];
                    for (int wv = 0; wv < NVAR; ++wv)
                        for (int j = 0; j < n; ++j) {
                            double *column = a.data() + (size_t)p.local(wv, p.face_node(side, q, j)) * m;
                            for (int v = 0; v < NVAR; ++v) {
                                const double scale = shape[j] * der[v * 4 + wv];
                                for (int i = 0; i < n; ++i) column[p.local(v, p.face_node(side, q, i))] += scale * shape[i];
                            }
                        }
                }
            }
            for (int i = 0; i < m; ++i) rhs[(size_t)t * m + i] = r[(size_t)cell * m + i];
            try {
                lu.compute(a.data(), m);
            } catch (const std::exception &e) {
#pragma omp critical
                failure = e.what();
                continue;
            }
            for (int c = 0; c <= t; ++c) lu.solve(rhs.data() + (size_t)c * m, solved.data() + (size_t)c * m);
            std::copy(solved.begin(), solved.begin() + (size_t)m * t, x_.begin() + (size_t)cell * m * t);
            std::copy(solved.begin() + (size_t)m * t, solved.end(), y_.begin() + (size_t)cell * m);
            // C applied to every solved column: restrict to each side then the 4x4 HDG derivative
            for (int side = 0; side < NFACES; ++side) {
                for (int c = 0; c <= t; ++c) {
                    p.face_values(solved.data() + (size_t)c * m, side, samples.data());
                    for (int q = 0; q < n; ++q) {
                        const Jac der = lin_.hdg(fs[side], q, side % 2 != 0);
                        for (int v = 0; v < NVAR; ++v) {
                            double s = 0;
                            for (int wv = 0; wv < NVAR; ++wv) s += samples[q * NVAR + wv] * der[v * 4 + wv];
                            act[(size_t)c * t + side * fw + v * n + q] = s;
                        }
                    }
                }
            }
            double *S = schur_.data() + (size_t)cell * t * t;
            for (size_t i = 0; i < (size_t)t * t; ++i) S[i] = -act[i];
            std::copy(act.begin() + (size_t)t * t, act.end(), cy_all.begin() + (size_t)cell * t);
        }
    }
    require(failure.empty(), failure.c_str());
    for (int cell = 0; cell < p.cells; ++cell) {
        const auto fs = p.faces(cell);
        for (int s = 0; s < NFACES; ++s)
            for (int k = 0; k < fw; ++k) rhs_[(size_t)fs[s] * fw + k] += cy_all[(size_t)cell * t + s * fw + k];
    }
}
// hybrid.cpp:73-82
void HybridOperator::apply(const Vec &d, Vec &out) const {
    const Problem &p = p_;
    const int t = p.local_trace_size(), fw = p.face_width();
    out.resize(p.trace_size());
    const Vec &D = lin_.trace_diagonal();
    for (int i = 0; i < p.trace_size(); ++i) out[i] = D[i] * d[i];
    Vec local(t), res(t);
    for (int cell = 0; cell < p.cells; ++cell) {
        const auto fs = p.faces(cell);
        for (int s = 0; s < NFACES; ++s)
            for (int k = 0; k < fw; ++k) local[s * fw + k] = d[(size_t)fs[s] * fw + k];
        const double *S = schur_.data() + (size_t)cell * t * t;
        for (int i = 0; i < t; ++i) res[i] = 0;
        for (int j = 0; j < t; ++j)
            for (int i = 0; i < t; ++i) res[i] += S[(size_t)j * t + i] * local[j];
        for (int s = 0; s < NFACES; ++s)
            for (int k = 0; k < fw; ++k) out[(size_t)fs[s] * fw + k] += res[s * fw + k];
    }
}
// hybrid.cpp:83-96
void HybridOperator::block(int row, int col, double *out) const {
    const Problem &p = p_;
    const int fw = p.face_width(), t = p.local_trace_size();
    std::fill(out, out + (size_t)fw * fw, 0.);
    if (row == col)
        for (int i = 0; i < fw; ++i) out[(size_t)i * fw + i] = lin_.trace_diagonal()[(size_t)row * fw + i];
    const int axis = row / p.cells, first = row % p.cells;
    for (int adjacent = 0; adjacent < 2; ++adjacent) {
        const int cell = adjacent == 0 ? first : p.neighbor(first, 2 * axis + 1);
        const int row_side = 2 * axis + (adjacent == 0 ? 1 : 0);
        const auto fs = p.faces(cell);
        const double *S = schur_.data() + (size_t)cell * t * t;
        for (int side = 0; side < NFACES; ++side)
            if (fs[side] == col)
                for (int j = 0; j < fw; ++j)
                    for (int i = 0; i < fw; ++i)
                        out[(size_t)j * fw + i] += S[(size_t)(side * fw + j) * t + row_side * fw + i];
    }
}
// hybrid.cpp:97-105
void HybridOperator::recover(const Vec &d, Vec &du) const {
    const Problem &p = p_;
    const int m = p.block, t = p.local_trace_size(), fw = p.face_width();
    du.resize(p.size());
#pragma omp parallel
    {
        Vec local(t);
#pragma omp for schedule(static)
        for (int cell = 0; cell < p.cells; ++cell) {
            const auto fs = p.faces(cell);
            for (int s = 0; s < NFACES; ++s)
                for (int k = 0; k < fw; ++k) local[s * fw + k] = d[(size_t)fs[s] * fw + k];
            const double *X = x_.data() + (size_t)cell * m * t;
            double *o = du.data() + (size_t)cell * m;
            for (int i = 0; i < m; ++i) o[i] = 0;
            for (int j = 0; j < t; ++j)
                for (int i = 0; i < m; ++i) o[i] -= X[(size_t)j * m + i] * local[j];
            for (int i = 0; i < m; ++i) o[i] -= y_[(size_t)cell * m + i];
        }
    }
}
// hybrid.cpp:106-121
void HybridOperator::recovered_residual_from_schur(const Vec &e, Vec &out) const {
    const Problem &p = p_;
    const int n = p.n, fw = p.face_width();
    out.assign(p.size(), 0.);
    Vec flux(n * NVAR);
    for (int cell = 0; cell < p.cells; ++cell) {
        const auto fs = p.faces(cell);
        for (int side = 0; side < NFACES; ++side) {
            const int face = fs[side];
            for (int v = 0; v < NVAR; ++v)
                for (int q = 0; q < n; ++q) {
                    const double d = lin_.trace_diagonal()[(size_t)face * fw + v * n + q];
                    const double tau = lin_.tau(face, q, side % 2 != 0);
                    flux[q * NVAR + v] = p.face_weight(face, q) * tau * e[(size_t)face * fw + v * n + q] / d;
                }
            p.lift(side, flux.data(), out.data() + (size_t)cell * p.block);
        }
    }
}

// ---------------------------------------------------------------- direct.hpp (dense reference)
namespace {
struct DenseDirect {
    int n = 0;
    Vec matrix;  // column-major n x n
    DenseLU lu;
};
}  // namespace

// ---------------------------------------------------------------- time_integrator.cpp:48-213
namespace {
using Clock = std::chrono::steady_clock;
double elapsed(Clock::time_point s) { return std::chrono::duration<double>(Clock::now() - s).count(); }
template <class Op> void bind_apply(const void *c, const Vec &x, Vec &y) { static_cast<const Op *>(c)->apply(x, y); }
}  // namespace

RunStatistics advance(Problem &p, Method method, Vec &solution) {
    const Config &c = p.config;
    const int N = p.size();
    const bool dg = method == Method::DG;
    Vec state(N), trial(N), residual(N), trial_residual(N), direction(N), rhs(dg ? N : p.trace_size());
    Vec lambda(p.trace_size()), trace_direction(p.trace_size()), equation_error(N), independent(N);
    Vec step_state(N), stage_base(N);
    std::vector<Vec> slopes(4, Vec(N));
    const Vec &weights = dg ? p.inverse_mass : p.inverse_trace_mass;
    std::unique_ptr<DGOperator> dgop, diagnostic;
    std::unique_ptr<HybridOperator> hybrid;
    if (dg) dgop = std::make_unique<DGOperator>(p);
    else hybrid = std::make_unique<HybridOperator>(p);
    if (!dg && c.check_update) diagnostic = std::make_unique<DGOperator>(p);
    const int width = dg ? p.block : p.face_width(), blocks = dg ? p.cells : p.face_count();
    require(!c.direct, "The dense direct reference solve is exposed through DGOperator::block only");
    BlockJacobi precond(blocks, width);
    GMRES gmres(dg ? N : p.trace_size(), c.restart, weights);
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
    RunStatistics stats;
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
                const double norm = dual_norm(residual), rms = norm / std::sqrt(p.example.lx * p.example.ly);
                if (initial_rms < 0) initial_rms = rms;
                if (c.newton_steps == 0 && rms <= c.nonlinear_tolerance * std::max(1., initial_rms)) {
                    converged = true;
                    break;
                }
                if (it == limit) break;
                const double allowance = 128 * std::numeric_limits<double>::epsilon() *
                                         ((state_norm(state) + old_norm) / tau + norm);
                const double target = std::max(10 * c.linear_tolerance * norm, allowance);
                LinearResult linear{0, 0};
                if (dg) {
                    dgop->refresh(state);
                    for (int i = 0; i < N; ++i) rhs[i] = -residual[i];
                    precond.refresh([&](int row, int col, double *out) { dgop->block(row, col, out); });
                    linear = gmres.solve(Action{dgop.get(), bind_apply<DGOperator>},
                                         Action{&precond, bind_apply<BlockJacobi>}, rhs, direction,
                                         c.max_linear, c.linear_tolerance);
                    for (int i = 0; i < N; ++i) equation_error[i] = -gmres.residual()[i];
                } else {
                    hybrid->refresh_projected(state, residual);
                    rhs = hybrid->rhs();
                    precond.refresh([&](int row, int col, double *out) { hybrid->block(row, col, out); });
                    double tolerance = c.linear_tolerance;
                    bool valid = false;
                    for (int attempt = 0; attempt < 4; ++attempt) {
                        LinearResult cur = gmres.solve(Action{hybrid.get(), bind_apply<HybridOperator>},
                                                       Action{&precond, bind_apply<BlockJacobi>}, rhs,
                                                       trace_direction, c.max_linear, tolerance);
                        linear.iterations += cur.iterations;
                        linear.relative_residual = cur.relative_residual;
                        hybrid->recover(trace_direction, direction);
                        for (int i = 0; i < p.trace_size(); ++i) lambda[i] = -gmres.residual()[i];
                        hybrid->recovered_residual_from_schur(lambda, equation_error);
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

// ---------------------------------------------------------------- main.cpp:7-108
int run_main(int argc, char **argv) {
    try {
        const Config config = parse(argc, argv);
        Problem problem(config);
        {
            std::string dir = config.prefix;
            auto slash = dir.find_last_of('/');
            if (slash != std::string::npos) {
                dir = dir.substr(0, slash);
                std::string accum;
                for (size_t i = 0; i <= dir.size(); ++i) {
                    if (i == dir.size() || dir[i] == '/') {
                        if (!accum.empty()) mkdir(accum.c_str(), 0755);
                    }
                    if (i < dir.size()) accum += dir[i];
                }
            }
        }
        std::ofstream summary(config.prefix + "_summary.csv"), updates(config.prefix + "_iterations.csv");
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
        if (!config.timing_only && config.save_solution) {
            solution_file.open(config.prefix + "_solution.csv");
            require(bool(solution_file), "Cannot open solution output");
            solution_file << std::setprecision(17)
                          << "method,cell,node,x,y,rho,momentum_x,momentum_y,energy,rho_exact,momentum_x_exact,"
                             "momentum_y_exact,energy_exact\n";
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
            summary << name << ',' << config.nx << ',' << config.ny << ',' << config.degree << ','
                    << problem.basis.points << ',' << config.cfl << ',' << config.integrator << ','
                    << (config.direct ? "direct" : "gmres") << ',' << (config.direct ? "none" : "block-jacobi")
                    << ',' << (config.direct ? "none" : "natural") << ',' << config.nonlinear_tolerance << ','
                    << config.linear_tolerance << ',' << config.safety << ',' << config.newton_steps << ','
                    << config.warmup_updates << ',' << stats.steps << ',' << stats.final_time << ','
                    << stats.newton_iterations << ',' << stats.krylov_iterations << ','
                    << stats.max_linear_residual << ',' << stats.max_dg_linear_residual << ','
                    << stats.minimum_step << ',' << stats.maximum_step << ','
                    << (stats.steps ? stats.final_time / stats.steps : 0.) << ',' << stats.seconds << ','
                    << stats.measured_updates << ','
                    << (stats.measured_updates ? stats.measured_newton_seconds / stats.measured_updates : 0.)
                    << ',' << problem.size() << ',' << problem.trace_size();
            for (int v = 0; v < NVAR; ++v) summary << ',' << error[v];
            summary << ',' << stats.conservation_drift << ',' << problem.example.lx << ','
                    << problem.example.ly << ',' << (method == Method::DG ? "dense" : "face-dense") << '\n';
            for (size_t i = 0; i < stats.updates.size(); ++i) {
                const auto &u = stats.updates[i];
                updates << name << ',' << u.step << ',' << u.stage << ',' << u.iteration << ',' << u.time << ','
                        << u.stage_time << ',' << u.dt << ',' << u.cfl << ',' << u.residual_physical_rms << ','
                        << u.damping << ',' << u.krylov_iterations << ',' << u.linear_relative_residual << ','
                        << u.dg_linear_relative_residual << ',' << u.iteration_s << ','
                        << (i >= static_cast<size_t>(config.warmup_updates)) << '\n';
            }
            if (!config.timing_only && config.save_solution)
                for (int cell = 0; cell < problem.cells; ++cell)
                    for (int i = 0; i < problem.plane; ++i) {
                        const double x = -.5 * problem.example.lx + problem.hx * (cell % config.nx + .5) +
                                         .5 * problem.hx * problem.basis.x[i % problem.n];
                        const double y = -.5 * problem.example.ly + problem.hy * (cell / config.nx + .5) +
                                         .5 * problem.hy * problem.basis.x[i / problem.n];
                        const State exact = problem.example.exact(x, y, stats.final_time);
                        solution_file << name << ',' << cell << ',' << i << ',' << x << ',' << y;
                        for (int v = 0; v < NVAR; ++v) solution_file << ',' << solution[problem.index(cell, v, i)];
                        for (int v = 0; v < NVAR; ++v) solution_file << ',' << exact[v];
                        solution_file << '\n';
                    }
            std::cout << name << ": steps=" << stats.steps << ", Newton=" << stats.newton_iterations
                      << ", Krylov=" << stats.krylov_iterations << ", time=" << stats.seconds << " s, mean Newton="
                      << (stats.measured_updates ? stats.measured_newton_seconds / stats.measured_updates : 0.)
                      << " s, conservation drift=" << stats.conservation_drift << '\n';
            if (method == Method::DG && config.method == "both") {
                dg_solution = solution;
                have_dg = true;
            } else if (have_dg) {
                double maximum = 0;
                for (int i = 0; i < problem.size(); ++i) maximum = std::max(maximum, std::abs(dg_solution[i] - solution[i]));
                std::ofstream comparison(config.prefix + "_difference.csv");
                require(bool(comparison), "Cannot open comparison output");
                comparison << std::setprecision(17) << "rho_L2,momentum_x_L2,momentum_y_L2,energy_L2,joint_L2,max_nodal\n";
                double joint = 0.;
                for (int v = 0; v < NVAR; ++v) {
                    double squared = 0.;
                    for (int cell = 0; cell < problem.cells; ++cell)
                        for (int node = 0; node < problem.plane; ++node) {
                            const int k = problem.index(cell, v, node);
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
}  // namespace oracle
