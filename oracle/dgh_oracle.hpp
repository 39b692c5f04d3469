// Test infrastructure only: the CPU oracle for the 2D DG / condensed-HDG Euler Newton update.
//
// This header declares a plain C++17 restatement (no Eigen) of the reference solver
// YueWu2002/DG_HDG_Euler_Cpp, directory dg_hdg_2d/ plus common/.  Only tests/, the
// smoke check in __graft_entry__.py and the cpu_baseline leg of bench.py may load it; the
// product library never links or calls it.  Every routine cites the reference file:line it
// restates.  Parity of this restatement is pinned against the reference's archived outputs
// (tests/golden/, produced by tests/golden/make_golden.py from the reference's result CSVs).
#pragma once
#include <array>
#include <cmath>
#include <cstdint>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace oracle {
using Vec = std::vector<double>;
constexpr int NDIM = 2, NVAR = 4, NFACES = 4;
enum Component { Density = 0, MomentumX = 1, MomentumY = 2, Energy = 3 };
using State = std::array<double, NVAR>;
using Jac = std::array<double, NVAR * NVAR>;  // row-major (v,w): d flux_v / d u_w

// types.hpp:18-21 — require() throws std::runtime_error with the given text.
inline void require(bool condition, const char *message) {
    if (!condition) throw std::runtime_error(message);
}

// config.hpp:7-18 — defaults identical to the reference.
struct Config {
    int nx = 8, ny = 8, degree = 3, quadrature = 0;
    int restart = 30, max_linear = 1500, max_newton = 30, steps = 0;
    int newton_steps = 0, warmup_updates = 0;
    double cfl = 2., final_time = .2, safety = 1.1;
    double nonlinear_tolerance = 1e-12, linear_tolerance = 1e-12;
    bool direct = false, colamd = false, timing_only = false, check_update = false,
         save_solution = true;
    std::string integrator = "ssp-dirk3";
    std::string method = "both", testcase = "diagonal", prefix = "output/run_2d";
};
Config parse(int argc, char **argv);  // config.cpp:31-122
void validate(const Config &c);       // config.cpp:6-22

// nodal_basis.hpp:9-66: Gauss nodes, and the volume quadrature of `points` >= nodes points.
struct Basis {
    int nodes = 0, points = 0;
    Vec x, w, left, right;
    Vec dw;  // weighted derivative at the nodes, dw[q*n+i] = w_q * l_i'(x_q)
    Vec qx, qw;      // volume rule (points)
    Vec values, wd;  // [q][i]: l_i(qx_q) (identity when points == nodes), qw_q * l_i'(qx_q)
    Vec ex, ew, evalues, projection;  // error rule, values [Q][n], projection [n][Q]
    explicit Basis(int degree, int quadrature = 0);
    Vec evaluate(double z) const;
};
void gauss(int n, Vec &x, Vec &w);

// physics.cpp:4-70
struct Gas {
    double gamma = 3.;
    double pressure(const State &u) const;
    void primitive(const State &u, double &inv_rho, double &vx, double &vy, double &p,
                   double &H) const;
    State flux(const State &u, int axis) const;
    Jac cached_jacobian(double u, double v, double H, int axis) const;
};
struct Speed { double a, b; };
Speed einfeldt(const State &l, const State &r, const Gas &gas, double safety, int axis);

// example.cpp:4-39
struct Example {
    Gas gas;
    std::string testcase;
    double cosine, sine, lx, ly;
    explicit Example(const std::string &name, double degrees = 45.);
    State exact(double x, double y, double t) const;
    double shock_time() const;
};

// discretization.hpp:7-45 / discretization.cpp
class Problem {
  public:
    Config config;
    Basis basis;
    int nx, ny, n, cells, plane, block;  // block = NVAR*n*n
    Example example;
    double hx, hy, step_size = 0;
    int Q = 0;  // volume quadrature points per direction (Q > n: over-integrated volume terms)
    Vec old, mass, inverse_mass, trace_mass, inverse_trace_mass;
    std::vector<Speed> speeds;
    explicit Problem(const Config &c);
    int size() const { return cells * block; }
    int index(int cell, int v, int node) const { return cell * block + v * plane + node; }
    int local(int v, int node) const { return v * plane + node; }
    int neighbor(int cell, int side) const;
    std::array<int, NFACES> faces(int cell) const;
    int face_width() const { return n * NVAR; }
    int face_count() const { return NDIM * cells; }
    int trace_size() const { return face_count() * face_width(); }
    int local_trace_size() const { return NFACES * face_width(); }
    double face_weight(int face, int q) const;
    int face_node(int side, int q, int i) const;
    // values[q*NVAR+v] = restriction of cell data (block-sized, var-major) to a side
    void face_values(const double *nodal, int side, double *values) const;
    void lift(int side, const double *values, double *nodal, double scale = 1) const;
    void initial(Vec &u) const;
    double freeze(const Vec &u);
    void trace(const Vec &u, Vec &lambda) const;
    void volume_residual(const Vec &u, Vec &r) const;
    void dg_residual(const Vec &u, Vec &r) const;
    void hybrid_residual(const Vec &u, const Vec &lambda, Vec &r, Vec &g) const;
    bool admissible(const Vec &u) const;
    double residual_norm(const Vec &r) const;
    State integral(const Vec &u) const;
    State error(const Vec &u, double time) const;

    // tensor_product.cpp:11-21: nodal cell data (var-major) -> values at the Q x Q points,
    // pts[v*Q*Q + qx + Q*qy]
    void interpolate(const double *nodal, double *pts) const;
    // tensor_product.cpp:57-72 (points != nodes): r -= (hy/2) Wd^T Fx (qw V) + (hx/2) (qw V)^T Fy Wd
    void subtract_weak_points(const double *fx, const double *fy, double *r) const;

  private:
    bool physical(const double *states_qv, int count) const;
    void subtract_weak(const double *fx, const double *fy, double *r) const;
};

// volume_jacobian.cpp + face_jacobian.cpp + dg_operator.cpp
class DGOperator {
  public:
    explicit DGOperator(const Problem &p);
    void refresh(const Vec &u);
    void apply(const Vec &d, Vec &out) const;
    void apply_transpose(const Vec &w, Vec &out) const;  // adjoint J^T w (test-side restatement)
    // Column-major block (as the reference's BlockRef): out[row + m*col]
    void block(int row, int col, double *out) const;
    // face Jacobian pieces shared with the hybrid operator
    Jac hll(int face, int q, bool left) const;
    Jac hdg(int face, int q, bool left) const;
    double tau(int face, int q, bool left) const;
    const Vec &trace_diagonal() const { return diagonal_; }
    const Problem &problem() const { return p_; }
    void volume_block(int cell, double *out) const;  // column-major m x m incl. mass/tau

  private:
    const Problem &p_;
    double inverse_step_ = 0;
    bool ready_ = false;
    Vec prim_;                   // [cell][point][3] = u, v, H at the volume points
    Vec fl_, fr_;                // [face][q][3]
    Vec tau_l_, tau_r_, blend_l_, blend_r_, penalty_, weights_;  // [face][q]
    Vec diagonal_;               // trace diagonal D
    Jac physical(int face, int q, bool left) const;
    void normal_action(const double *prim, const double *d, double *out, int axis) const;
};

// dense_lu.hpp / block_jacobi.hpp — own row-partial-pivot LU (first maximum wins ties).
struct DenseLU {
    int m = 0;
    Vec lu;                  // column-major
    std::vector<int> perm;   // P: (P b)[i] = b[perm[i]]
    void compute(const double *a, int width);   // throws on non-finite / singular
    void solve(const double *b, double *x) const;  // x may alias b
    void right_solve(double *x) const;             // X <- X A^{-1}, X column-major m x m
};
// block_ilu.cpp:15-84 with the natural ordering (block_graph.cpp:7-19 pattern: each row's
// columns sorted, the diagonal included): the ILU(0) kind of BlockPreconditioner.  Blocks are
// column-major width x width; the provider fills block (row, col).
class BlockILU0 {
  public:
    BlockILU0(const std::vector<std::vector<int>> &adjacency, int width);
    void refresh(const std::function<void(int, int, double *)> &provider);
    void apply(const Vec &rhs, Vec &result) const;
    int rows, width;
    std::vector<int> row_ptr, col_idx, diag;
    std::vector<int> upd_off, upd_target, upd_upper;  // block_ilu.cpp:24-45 symbolic schedule
    Vec values;
    std::vector<DenseLU> lus;
    double *block(int slot) { return &values[(size_t)slot * width * width]; }
    const double *block(int slot) const { return &values[(size_t)slot * width * width]; }
    int find(int row, int col) const;
};
// BlockGraph::periodic(cells) adjacency (block_graph.cpp:30-35)
std::vector<std::vector<int>> periodic_adjacency(int cells);
// BlockGraph::cartesian(nx, ny) adjacency (block_graph.cpp:20-29): each cell, its left, right,
// lower and upper periodic neighbours, cells numbered x + nx y.
std::vector<std::vector<int>> cartesian_adjacency(int nx, int ny);
class BlockJacobi {
  public:
    BlockJacobi(int blocks, int width);
    void refresh(const std::function<void(int, int, double *)> &provider);
    void apply(const Vec &rhs, Vec &result) const;
    int blocks, width;
    std::vector<DenseLU> lus;
};

// gmres.hpp / gmres.cpp
struct LinearResult { int iterations; double relative_residual; };
using ActionFn = void (*)(const void *, const Vec &, Vec &);
struct Action {
    const void *context;
    ActionFn call;
    void operator()(const Vec &x, Vec &y) const { call(context, x, y); }
};
class GMRES {
  public:
    GMRES(int size, int restart, const Vec &weights);
    LinearResult solve(Action A, Action M, const Vec &rhs, Vec &x, int limit, double tol);
    const Vec &residual() const { return residual_; }

  private:
    int n_, restart_;
    std::vector<Vec> basis_;
    Vec h_, cosine_, sine_, g_, y_, work_, residual_, column_, weights_, proj_;
    double dot(const Vec &a, const Vec &b) const;
    double norm(const Vec &a) const;
};

// hybrid.cpp
class HybridOperator {
  public:
    explicit HybridOperator(const Problem &p);
    void refresh_projected(const Vec &u, const Vec &r);
    void apply(const Vec &d, Vec &out) const;
    void block(int row, int col, double *out) const;  // column-major fw x fw
    void recover(const Vec &dlambda, Vec &du) const;
    void recovered_residual_from_schur(const Vec &e, Vec &out) const;
    const Vec &rhs() const { return rhs_; }
    const Vec &schur() const { return schur_; }  // [cell][t][t] column-major per cell
    const Vec &xpool() const { return x_; }      // [cell] m x t column-major
    const Vec &ypool() const { return y_; }      // [cell][m]
    const DGOperator &linearisation() const { return lin_; }

  private:
    const Problem &p_;
    DGOperator lin_;
    Vec x_, schur_, y_, rhs_;
};

// time_integrator.hpp:9-20
struct UpdateStatistics {
    int step, stage, iteration, krylov_iterations;
    double time, stage_time, dt, cfl, residual_physical_rms, damping;
    double linear_relative_residual, dg_linear_relative_residual, iteration_s;
};
struct RunStatistics {
    double final_time = 0, conservation_drift = 0, seconds = 0, max_linear_residual = 0;
    double max_dg_linear_residual = 0, minimum_step = 0, maximum_step = 0;
    double measured_newton_seconds = 0;
    int steps = 0, newton_iterations = 0, krylov_iterations = 0, measured_updates = 0;
    std::vector<UpdateStatistics> updates;
};
enum class Method { DG, HDG };
RunStatistics advance(Problem &p, Method method, Vec &solution);  // time_integrator.cpp:48-213
int run_main(int argc, char **argv);                               // main.cpp:7-108
void set_threads(int threads);
}  // namespace oracle
