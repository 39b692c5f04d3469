// Exact rotated simple wave / entropy wave (example.cpp:4-39), the projected initial state with
// positivity scaling (initial_and_error.cpp:4-54) and the L2 error (initial_and_error.cpp:55-73),
// on the max(20, 2n+3)-point Gauss rule per direction.
#pragma once
#include "dgh_common.cuh"

namespace dgh {

constexpr int MAXQ = 21;

struct Case {
    int kind;  // 0 diagonal (rotated 45 deg), 1 wave (entropy), 2 axis
    double cosine, sine, lx, ly, gamma;
};

// Error rule and its tables, passed by pointer (device buffer): ex, ew [Q], ev [Q][N] (Lagrange
// values at ex), proj [N][Q] = diag(1/w) ev^T diag(ew).
struct ErrorRule {
    int Q;
    double ex[MAXQ], ew[MAXQ], ev[MAXQ * MAXN], proj[MAXN * MAXQ];
};

__device__ inline bool exact_state(const Case &c, double x, double y, double t, double u[4]) {
    const double g = c.gamma, pi = 3.14159265358979323846;
    if (c.kind == 1) {
        const double rho = 1 + .2 * sin(pi * (x - t)) * sin(pi * (y - .5 * t));
        u[0] = rho; u[1] = rho; u[2] = .5 * rho; u[3] = 1 / (g - 1) + .625 * rho;
        return true;
    }
    const bool ok = t < 4 / ((g + 1) * pi);
    const bool diagonal = c.kind == 0;
    if (diagonal) x = c.cosine * x + c.sine * y;
    const double a = (3 - g) / 2, b = (g + 1) / 4;
    double lo = x - t * (a + b), hi = x - t * (a - b), xi = x - t * a;
    for (int it = 0; it < 80; ++it) {
        const double f = xi + t * (a + b * sin(pi * xi)) - x;
        if (fabs(f) < 2e-15) break;
        if (f > 0) hi = xi; else lo = xi;
        const double z = xi - f / (1 + t * b * pi * cos(pi * xi));
        xi = z > lo && z < hi ? z : .5 * (lo + hi);
    }
    const double jm = sin(pi * xi), velocity = .5 * (2 + jm), sound = (g - 1) * (2 - jm) / 4;
    const double rho = pow(sound * sound / g, 1 / (g - 1));
    u[0] = rho;
    u[1] = rho * velocity * (diagonal ? c.cosine : 1.);
    u[2] = diagonal ? rho * velocity * c.sine : 0.;
    u[3] = pow(rho, g) / (g - 1) + .5 * rho * velocity * velocity;
    return ok;
}

template <int N>
__global__ void __launch_bounds__(256)
k_initial(double *__restrict__ u, const ErrorRule *__restrict__ er, Basis1D b, Grid g, Case c, int *status) {
    constexpr int P = N * N;
    const int Q = er->Q;
    __shared__ double S[MAXQ * MAXQ * NVAR];
    __shared__ double scr[NVAR * MAXN * MAXQ];
    __shared__ double U[NVAR * P];
    __shared__ double chk[(2 * P + MAXQ * MAXQ + NFACES * N) * NVAR];
    __shared__ double mean[NVAR];
    const int cell = blockIdx.x, cx = cell % g.nx, cy = cell / g.nx + g.row0;
    for (int k = threadIdx.x; k < Q * Q; k += blockDim.x) {
        const int i = k % Q, j = k / Q;
        double s[4];
        const bool ok = exact_state(c, -.5 * c.lx + g.hx * (cx + .5) + .5 * g.hx * er->ex[i],
                                    -.5 * c.ly + g.hy * (cy + .5) + .5 * g.hy * er->ex[j], 0., s);
        if (!ok) atomicOr(status, ST_SHOCK);
#pragma unroll
        for (int v = 0; v < NVAR; ++v) S[k * NVAR + v] = s[v];
    }
    __syncthreads();
    // scratch(a, j) = sum_i proj(a, i) S(i, j); U(a, bb) = sum_j scratch(a, j) proj(bb, j)
    for (int k = threadIdx.x; k < NVAR * N * Q; k += blockDim.x) {
        const int v = k / (N * Q), a = (k / Q) % N, j = k % Q;
        double s = 0;
        for (int i = 0; i < Q; ++i) s += er->proj[a * Q + i] * S[(i + Q * j) * NVAR + v];
        scr[k] = s;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < NVAR * P; k += blockDim.x) {
        const int v = k / P, a = (k % P) % N, bb = (k % P) / N;
        double s = 0;
        for (int j = 0; j < Q; ++j) s += scr[(v * N + a) * Q + j] * er->proj[bb * Q + j];
        U[k] = s;
    }
    __syncthreads();
    if (threadIdx.x < NVAR) {
        const int v = threadIdx.x;
        double s = 0;
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < N; ++i) s += .25 * b.w[i] * b.w[j] * U[v * P + i + N * j];
        mean[v] = s;
    }
    // check points: nodes twice (collocated volume points), error points, four sides
    for (int k = threadIdx.x; k < 2 * P; k += blockDim.x)
        for (int v = 0; v < NVAR; ++v) chk[k * NVAR + v] = U[v * P + k % P];
    for (int k = threadIdx.x; k < Q * Q; k += blockDim.x) {
        const int qi = k % Q, qj = k / Q;
        for (int v = 0; v < NVAR; ++v) {
            double s = 0;
            for (int bb = 0; bb < N; ++bb)
                for (int a = 0; a < N; ++a) s += er->ev[qi * N + a] * er->ev[qj * N + bb] * U[v * P + a + N * bb];
            chk[(2 * P + k) * NVAR + v] = s;
        }
    }
    for (int k = threadIdx.x; k < NFACES * N; k += blockDim.x) {
        const int side = k / N, q = k % N;
        const double *e = side % 2 ? b.eR : b.eL;
        for (int v = 0; v < NVAR; ++v) {
            double s = 0;
            for (int i = 0; i < N; ++i) s += e[i] * U[v * P + face_node(N, side, q, i)];
            chk[(2 * P + Q * Q + k) * NVAR + v] = s;
        }
    }
    __syncthreads();
    __shared__ double theta_s;
    if (threadIdx.x == 0) {
        double m[4] = {mean[0], mean[1], mean[2], mean[3]};
        if (!(m[0] > 0 && pressure(g.gamma, m) > 0)) atomicOr(status, ST_NONPHYS_MEAN);
        double theta = 1;
        const int count = 2 * P + Q * Q + NFACES * N;
        for (int q = 0; q < count; ++q) {
            double d[4];
            for (int v = 0; v < NVAR; ++v) d[v] = chk[q * NVAR + v] - m[v];
            auto phys = [&](double f) {
                double z[4];
                for (int v = 0; v < NVAR; ++v) z[v] = m[v] + f * d[v];
                return z[0] > 1e-12 && pressure(g.gamma, z) > 1e-12;
            };
            if (!phys(theta)) {
                double low = 0, high = theta;
                for (int it = 0; it < 60; ++it) {
                    const double mid = .5 * (low + high);
                    if (phys(mid)) low = mid; else high = mid;
                }
                theta = .99 * low;
            }
        }
        theta_s = theta;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < NVAR * P; k += blockDim.x) {
        const int v = k / P;
        u[(size_t)cell * NVAR * P + k] = mean[v] + theta_s * (U[k] - mean[v]);
    }
}

// partial[cell*4 + v] = sum over the error points of .25 hx hy ew_i ew_j (u_h - u_exact)^2
template <int N>
__global__ void __launch_bounds__(256)
k_l2_error(const double *__restrict__ u, const ErrorRule *__restrict__ er, Basis1D b, Grid g, Case c, double t,
           double *__restrict__ partial, int *status) {
    constexpr int P = N * N;
    const int Q = er->Q;
    __shared__ double U[NVAR * P];
    __shared__ double red[4][256];
    const int cell = blockIdx.x, cx = cell % g.nx, cy = cell / g.nx + g.row0;
    for (int k = threadIdx.x; k < NVAR * P; k += blockDim.x) U[k] = u[(size_t)cell * NVAR * P + k];
    __syncthreads();
    double acc[4] = {0, 0, 0, 0};
    for (int k = threadIdx.x; k < Q * Q; k += blockDim.x) {
        const int i = k % Q, j = k / Q;
        double e[4];
        if (!exact_state(c, -.5 * c.lx + g.hx * (cx + .5) + .5 * g.hx * er->ex[i],
                         -.5 * c.ly + g.hy * (cy + .5) + .5 * g.hy * er->ex[j], t, e))
            atomicOr(status, ST_SHOCK);
        for (int v = 0; v < NVAR; ++v) {
            double s = 0;
            for (int bb = 0; bb < N; ++bb)
                for (int a = 0; a < N; ++a) s += er->ev[i * N + a] * er->ev[j * N + bb] * U[v * P + a + N * bb];
            const double d = s - e[v];
            acc[v] += .25 * g.hx * g.hy * er->ew[i] * er->ew[j] * d * d;
        }
    }
    for (int v = 0; v < 4; ++v) red[v][threadIdx.x] = acc[v];
    __syncthreads();
    if (threadIdx.x < 4) {
        double s = 0;
        for (int k = 0; k < (int)blockDim.x; ++k) s += red[threadIdx.x][k];
        partial[(size_t)cell * 4 + threadIdx.x] = s;
    }
}

// conservation integrals: partial[cell*4+v] = sum_node u * mass
template <int N>
__global__ void k_integral(const double *__restrict__ u, Basis1D b, Grid g, double *__restrict__ partial) {
    constexpr int P = N * N;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= g.cells * NVAR) return;
    const int cell = idx / NVAR, v = idx % NVAR;
    double s = 0;
    for (int node = 0; node < P; ++node)
        s += u[(size_t)cell * NVAR * P + v * P + node] * (.25 * g.hx * g.hy * b.w[node % N] * b.w[node / N]);
    partial[idx] = s;
}

}  // namespace dgh
