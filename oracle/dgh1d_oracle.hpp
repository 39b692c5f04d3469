// Test infrastructure only: the CPU oracle for the 1D DG / condensed-HDG Euler Newton update.
//
// A plain C++17 restatement (no Eigen) of the reference solver's 1D program, directory
// dg_hdg_1d/ of YueWu2002/DG_HDG_Euler_Cpp, with the shared linear algebra (dense LU, GMRES)
// taken from the 2D oracle in dgh_oracle.hpp.  Only tests/ and the smoke check load it; the
// product library never links or calls it.  Parity is pinned against the reference's archived
// 1D runs (code_test/1d/results, accuracy_test/results/1d_*), copied into tests/golden/.
#pragma once
#include "dgh_oracle.hpp"

namespace oracle1d {
using oracle::require;
using Vec = std::vector<double>;
constexpr int NVAR = 3, NFACES = 2;
enum Component { Density = 0, Momentum = 1, Energy = 2 };
using State = std::array<double, NVAR>;
using Jac = std::array<double, NVAR * NVAR>;  // row-major (v,w): d flux_v / d u_w

// dg_hdg_1d/include/euler/config.hpp:7-19 — defaults identical to the reference.
struct Config {
    int cells = 32, degree = 3, quadrature = 0;
    int restart = 30, max_linear = 1500, max_newton = 30, steps = 0;
    int newton_steps = 0, warmup_updates = 0;
    double cfl = 2., final_time = .2, safety = 1.1;
    double nonlinear_tolerance = 1e-12, linear_tolerance = 1e-12;
    bool ilu = false, direct = false, colamd = false, timing_only = false, check_update = false;
    std::string integrator = "ssp-dirk3";
    std::string method = "both", prefix = "output/run";
};
Config parse(int argc, char **argv);  // dg_hdg_1d/src/config.cpp:29-114
void validate(const Config &c);       // dg_hdg_1d/src/config.cpp:6-28

// common/include/euler/nodal_basis.hpp:9-66 with a separate quadrature rule (over-integration).
struct Basis {
    int nodes = 0, points = 0;
    Vec x, w, qx, qw, left, right;
    Vec values;    // [Q][n] Lagrange values at the quadrature points (identity when Q == n)
    Vec wd;        // [Q][n] qw_q * l_i'(qx_q): the weighted derivatives
    Vec ex, ew, evalues, projection;  // error rule, its values [Qe][n], projection [n][Qe]
    Basis(int degree, int quadrature);
    Vec evaluate(double z) const;
};

// dg_hdg_1d/src/physics.cpp:4-38
struct Gas {
    double gamma = 3.;
    double pressure(const State &u) const;
    State flux(const State &u) const;
    Jac jacobian(const State &u) const;
    double spectral_radius(const State &u) const;
};
struct Speed { double a, b; };
Speed einfeldt(const State &l, const State &r, const Gas &gas, double safety);

// dg_hdg_1d/src/simple_wave.cpp:4-26, simple_wave.hpp:5-9
struct SimpleWave {
    Gas gas;
    State exact(double x, double t) const;
    double shock_time() const;
};

// dg_hdg_1d/include/euler/discretization.hpp / src/discretization.cpp
class Problem {
  public:
    Config config;
    SimpleWave example;
    Basis basis;
    int cells, n, block;  // block = NVAR * n, layout [cell][var][node] (types.hpp:82-108)
    double h, step_size = 0;
    Vec old, mass, inverse_mass;
    std::vector<Speed> speeds;  // one (a, b) per face; face e joins cells e and e+1
    explicit Problem(const Config &c);
    int size() const { return cells * block; }
    int index(int cell, int v, int i) const { return cell * block + v * n + i; }
    int local(int v, int i) const { return v * n + i; }
    State sample(const Vec &u, int cell, const Vec &shape) const;
    State quadrature_state(const Vec &u, int cell, int q) const;
    void initial(Vec &u) const;
    double freeze(const Vec &u);
    void trace(const Vec &u, Vec &lambda) const;
    void volume_residual(const Vec &u, Vec &r) const;
    void dg_residual(const Vec &u, Vec &r) const;
    bool admissible(const Vec &u) const;
    double residual_norm(const Vec &r) const;
    State integral(const Vec &u) const;
    State error(const Vec &u, double time) const;
};

// dg_hdg_1d/src/volume_jacobian.cpp
class VolumeJacobian {
  public:
    explicit VolumeJacobian(const Problem &p) : p_(p) {}
    void refresh(const Vec &u);
    void apply(const Vec &d, Vec &out) const;
    void block(int cell, double *out) const;  // column-major block x block

  private:
    const Problem &p_;
    std::vector<Jac> coef_;  // [cell][q]
    double inverse_step_ = 0;
    bool ready_ = false;
};

// dg_hdg_1d/src/dg_operator.cpp
class DGOperator {
  public:
    explicit DGOperator(const Problem &p) : p_(p), volume_(p) {}
    void refresh(const Vec &u);
    void apply(const Vec &d, Vec &out) const;
    void block(int row, int col, double *out) const;  // column-major

  private:
    const Problem &p_;
    VolumeJacobian volume_;
    std::vector<Jac> left_, right_;  // per face
    bool ready_ = false;
};

// dg_hdg_1d/src/hybrid.cpp
class HybridOperator {
  public:
    explicit HybridOperator(const Problem &p);
    void refresh_projected(const Vec &u, const Vec &r);
    void apply(const Vec &x, Vec &y) const;
    void block(int row, int col, double *out) const;  // column-major NVAR x NVAR
    void recover(const Vec &dl, Vec &du) const;
    void recovered_residual(const Vec &dl, Vec &out) const;
    const Vec &rhs() const { return rhs_; }

  private:
    struct Cell {
        Vec B, C, X, S, y;  // column-major: B m x 6, C 6 x m, X m x 6, S 6 x 6
    };
    const Problem &p_;
    VolumeJacobian volume_;
    std::vector<Cell> cells_;
    Vec rhs_;
    int face_index(int cell, int side) const;
};

// dg_hdg_1d/src/time_integrator.cpp:45-206 (GMRES with block Jacobi)
enum class Method { DG, HDG };
oracle::RunStatistics advance(Problem &p, Method method, Vec &solution);
int run_main(int argc, char **argv);  // dg_hdg_1d/src/main.cpp:7-107
}  // namespace oracle1d
