// Shared device code for the B200 DG / condensed-HDG Euler kernels.
//
// Layout contract (dg_hdg_2d/include/euler/types.hpp:22-31): a volume vector holds, per cell
// (x fastest, then y), NVAR sheets of n*n nodal values with the x node index fastest.  A trace
// vector holds per face (x-normal faces 0..E-1, then y-normal faces E..2E-1) NVAR lines of n
// values (discretization.cpp:65-68).  Face f < E is the +x side of cell f; face E+c is the +y
// side of cell c (discretization.cpp:78-80).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace dgh {

constexpr int NVAR = 4;
constexpr int NFACES = 4;
constexpr int MAXN = 9;

// Explicitly rounded arithmetic.  The compiler never fuses these into FMAs of its own choosing,
// so a kernel body written with them computes the same bits in every kernel it is inlined into
// (the single-problem kernels and the batched kernels of a lockstep batch share their bodies).
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// Status bits raised by kernels; the host maps each to the reference's require() text.
enum StatusBits : int {
    ST_FROZEN_FACE = 1 << 0,   // "Invalid frozen face state"          physics.cpp:108-109
    ST_CFL_VOLUME = 1 << 1,    // "Invalid CFL volume state"           discretization.cpp:233
    ST_SINGULAR = 1 << 2,      // "Singular block Jacobi factor"       block_jacobi.hpp:16-18
    ST_LU_INPUT = 1 << 3,      // "Nonfinite block LU input"           dense_lu.hpp:12
    ST_NONPHYS_MEAN = 1 << 4,  // "Nonphysical cell average"           initial_and_error.cpp:25
    ST_SHOCK = 1 << 5,         // "Simple wave reaches shock time"     example.cpp:19
    ST_SINGULAR_HDG = 1 << 6,  // "Singular or nonfinite LU factors"   dense_lu.hpp:15-16
};

// One-dimensional reference element on n Gauss nodes (nodal_basis.hpp:34-65), passed by value.
struct Basis1D {
    double w[MAXN];        // Gauss weights
    double eL[MAXN];       // Lagrange values at -1
    double eR[MAXN];       // Lagrange values at +1
    double dw[MAXN * MAXN];  // dw[q*n+i] = w_q l_i'(x_q)
};

// Geometry and the frozen stage scalars shared by most kernels.
struct Grid {
    int nx, ny, cells;
    double hx, hy;
    double gamma;
    int row0;  // global row of local row 0 (a slab of a decomposed mesh; 0 for the whole mesh)
};

__host__ __device__ inline int neighbor(const Grid &g, int cell, int side) {
    int x = cell % g.nx, y = cell / g.nx;
    if (side < 2) x = (x + (side == 0 ? g.nx - 1 : 1)) % g.nx;
    else y = (y + (side == 2 ? g.ny - 1 : 1)) % g.ny;
    return x + g.nx * y;
}
// faces(cell)[side] (discretization.cpp:78-80)
__host__ __device__ inline int face_of(const Grid &g, int cell, int side) {
    switch (side) {
        case 0: return neighbor(g, cell, 0);
        case 1: return cell;
        case 2: return g.cells + neighbor(g, cell, 2);
        default: return g.cells + cell;
    }
}
// face_node(side, tangent q, normal i) (discretization.cpp:84-86)
__host__ __device__ inline int face_node(int n, int side, int q, int i) {
    return side < 2 ? i + n * q : q + n * i;
}
__host__ __device__ inline double face_weight(const Grid &g, const Basis1D &b, int face, int q) {
    return .5 * (face < g.cells ? g.hy : g.hx) * b.w[q];
}

// ---- physics.cpp:4-70 ----------------------------------------------------------------------
struct Prim { double ir, vx, vy, p, H; };
__device__ inline Prim primitive(double gamma, const double u[4]) {
    Prim r;
    r.ir = 1. / u[0];
    r.vx = u[1] * r.ir;
    r.vy = u[2] * r.ir;
    r.p = (gamma - 1) * (u[3] - .5 * (u[1] * r.vx + u[2] * r.vy));
    r.H = (u[3] + r.p) * r.ir;
    return r;
}
__device__ inline double pressure(double gamma, const double u[4]) {
    return (gamma - 1) * (u[3] - .5 * (u[1] * u[1] + u[2] * u[2]) / u[0]);
}
__device__ inline void flux(double gamma, const double u[4], int axis, double f[4]) {
    const Prim p = primitive(gamma, u);
    const double va = axis == 0 ? p.vx : p.vy;
    f[0] = u[1 + axis];
    f[1] = u[1] * va;
    f[2] = u[2] * va;
    f[1 + axis] += p.p;
    f[3] = (u[3] + p.p) * va;
}
// Gas::cached_jacobian (physics.cpp:33-48): a[v*4+w] = dF_v/du_w from (u, v, H).
__device__ inline void cached_jacobian(double gamma, double u, double v, double H, int axis, double a[16]) {
    const double gm = gamma - 1., s2 = u * u + v * v;
#pragma unroll
    for (int i = 0; i < 16; ++i) a[i] = 0.;
    if (axis == 0) {
        a[1] = 1.;
        a[4] = .5 * (gamma - 3) * u * u + .5 * gm * v * v; a[5] = (3 - gamma) * u; a[6] = -gm * v; a[7] = gm;
        a[8] = -u * v; a[9] = v; a[10] = u; a[11] = 0.;
        a[12] = u * (.5 * gm * s2 - H); a[13] = H - gm * u * u; a[14] = -gm * u * v; a[15] = gamma * u;
    } else {
        a[2] = 1.;
        a[4] = -u * v; a[5] = v; a[6] = u; a[7] = 0.;
        a[8] = .5 * gm * u * u + .5 * (gamma - 3) * v * v; a[9] = -gm * u; a[10] = (3 - gamma) * v; a[11] = gm;
        a[12] = v * (.5 * gm * s2 - H); a[13] = -gm * u * v; a[14] = H - gm * v * v; a[15] = gamma * v;
    }
}
// Linearised normal flux dF(u,v,H)·d (volume_jacobian.cpp:43-58, face_jacobian.cpp:38-55).
__device__ inline void normal_action(double gamma, double u, double v, double H, const double d[4], int axis,
                                     double out[4]) {
    const double dr = d[0], dx = d[1], dy = d[2], de = d[3];
    const double dp = (gamma - 1.) * (de - u * dx - v * dy + .5 * (u * u + v * v) * dr);
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
// Einfeldt HLL bounds with safety factor (physics.cpp:49-69).  Returns false when a side state
// is not physical (the reference throws "Invalid frozen face state").
__device__ inline bool einfeldt(double gamma, const double l[4], const double r[4], double safety, int axis,
                                double &a, double &b) {
    const Prim pl = primitive(gamma, l), pr = primitive(gamma, r);
    const bool ok = l[0] > 0 && r[0] > 0 && pl.p > 0 && pr.p > 0;
    const double sl = sqrt(l[0]), sr = sqrt(r[0]);
    const double vx = (sl * pl.vx + sr * pr.vx) / (sl + sr), vy = (sl * pl.vy + sr * pr.vy) / (sl + sr);
    const double H = (sl * pl.H + sr * pr.H) / (sl + sr);
    const double sound = sqrt((gamma - 1) * (H - .5 * (vx * vx + vy * vy)));
    const double cl = sqrt(gamma * pl.p * pl.ir), cr = sqrt(gamma * pr.p * pr.ir);
    const double vla = axis == 0 ? pl.vx : pl.vy, vra = axis == 0 ? pr.vx : pr.vy, va = axis == 0 ? vx : vy;
    a = safety * fmax(fmax(0., -vla + cl), -va + sound);
    b = safety * fmax(fmax(0., vra + cr), va + sound);
    return ok;
}

// Block-wide deterministic sum of one double per thread (fixed reduction tree).
template <int THREADS>
__device__ inline double block_sum(double v, double *scratch) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    double r = 0;
    if (warp == 0) {
        r = lane < THREADS / 32 ? scratch[lane] : 0.;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    __syncthreads();
    return r;  // valid in thread 0
}

}  // namespace dgh
