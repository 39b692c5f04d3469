// An allocation-free form of the DG residual R(u) (see dgh_residual_noalloc in dgh_gpu.h).
//
// Some callers cannot allocate device memory: an allocation-free time loop (the reference
// requires exactly that of its own Newton updates), code that runs while a stream is being
// captured into a CUDA graph, where cudaMalloc is not permitted, or hosts that pre-plan every
// byte of device memory.  This entry point therefore takes its one piece of scratch memory, the
// per-cell face restrictions of u, from a fixed array that the library itself reserves at load
// time, and it allocates nothing, neither with cudaMalloc nor through any allocating library.
#include "dgh_gpu.h"
#include "dgh_kernels_dg.cuh"

#include <cmath>
#include <cstdio>
#include <mutex>

using namespace dgh;

namespace {
// Scratch for the face restrictions of u: 16 (k+1) doubles per cell.  Every GPU that loads the
// library holds these 16 MiB until the process exits.
constexpr long long kTraceCapacity = DGH_NOALLOC_TRACE_CAPACITY;
__device__ __align__(256) double g_noalloc_traces[kTraceCapacity];

// Device address of g_noalloc_traces per device, looked up once with that device current.
constexpr int kMaxDevices = 64;
double *g_trace_ptr[kMaxDevices] = {};
std::mutex g_setup_mutex;

void message(char *buf, int len, const char *text) {
    if (buf && len > 0) std::snprintf(buf, (size_t)len, "%s", text);
}

// Gauss-Legendre nodes and weights on fixed-size arrays (no heap), ascending nodes.
void gauss_fixed(int n, double *x, double *w) {
    const double pi = std::acos(-1.);
    for (int k = 0; k < (n + 1) / 2; ++k) {
        long double z = std::cos(pi * (k + .75) / (n + .5)), p0 = 1, p1 = z, dp = 1;
        for (int it = 0; it < 101; ++it) {
            p0 = 1;
            p1 = z;
            for (int j = 2; j <= n; ++j) {
                const long double p2 = ((2 * j - 1) * z * p1 - (j - 1) * p0) / j;
                p0 = p1;
                p1 = p2;
            }
            if (n == 1) { p1 = z; p0 = 1; }
            dp = n * (z * p1 - p0) / (z * z - 1);
            if (it == 100) break;
            const long double dz = p1 / dp;
            z -= dz;
            if (std::fabs((double)dz) <= 1e-19) it = 99;  // one more evaluation at the final z
        }
        x[n - 1 - k] = (double)z;
        x[k] = -(double)z;
        w[k] = w[n - 1 - k] = (double)(2 / ((1 - z * z) * dp * dp));
    }
    if (n % 2) x[n / 2] = 0;
}

// Weighted derivative and boundary values of the nodal basis (nodal_basis.hpp:34-65).
void basis_fixed(int n, Basis1D &b) {
    double x[MAXN], w[MAXN], bary[MAXN], D[MAXN * MAXN];
    gauss_fixed(n, x, w);
    for (int i = 0; i < n; ++i) {
        bary[i] = 1.;
        for (int j = 0; j < n; ++j)
            if (i != j) bary[i] /= x[i] - x[j];
    }
    for (int i = 0; i < n; ++i) {
        double s = 0;
        for (int j = 0; j < n; ++j)
            if (i != j) {
                D[i * n + j] = bary[j] / (bary[i] * (x[i] - x[j]));
                s += D[i * n + j];
            }
        D[i * n + i] = -s;
    }
    for (int i = 0; i < n; ++i) {
        double l = 1., r = 1.;
        for (int j = 0; j < n; ++j)
            if (i != j) {
                l *= (-1. - x[j]) / (x[i] - x[j]);
                r *= (1. - x[j]) / (x[i] - x[j]);
            }
        b.w[i] = w[i];
        b.eL[i] = l;
        b.eR[i] = r;
    }
    for (int q = 0; q < n; ++q)
        for (int i = 0; i < n; ++i) b.dw[q * n + i] = w[q] * D[q * n + i];
}

template <int N>
cudaError_t launch(const Grid &g, const Basis1D &b, double inv_step, const double *u, const double *old,
                   const double *speeds, double *r, double *traces, cudaStream_t stream) {
    using T = Team<N>;
    const int blocks = (g.cells + T::CPB - 1) / T::CPB;
    k_face_trace<N, false><<<blocks, T::THREADS, 0, stream>>>(u, traces, b, g, nullptr);
    k_residual<N><<<blocks, T::THREADS, 0, stream>>>(u, old, traces, speeds, r, b, g, inv_step);
    return cudaGetLastError();
}
}  // namespace

extern "C" int dgh_residual_noalloc(int nx, int ny, int degree, int testcase, double step_size, const double *u,
                                    const double *old, const double *speeds, double *r, void *stream, char *errbuf,
                                    int errbuf_len) {
    message(errbuf, errbuf_len, "");
    if (nx < 3 || ny < 3 || degree < 0 || degree > 8) {
        message(errbuf, errbuf_len, "Invalid mesh or degree");
        return DGH_ERR_INVALID;
    }
    if (testcase < DGH_TEST_DIAGONAL || testcase > DGH_TEST_AXIS || !(step_size > 0) || !std::isfinite(step_size)) {
        message(errbuf, errbuf_len, "Invalid testcase or step size");
        return DGH_ERR_INVALID;
    }
    if (!u || !old || !speeds || !r) {
        message(errbuf, errbuf_len, "null device pointer");
        return DGH_ERR_INVALID;
    }
    const int n = degree + 1;
    const long long need = (long long)nx * ny * NFACES * n * NVAR;
    if (need > kTraceCapacity) {
        char text[160];
        std::snprintf(text, sizeof text,
                      "mesh too large for the fixed scratch: needs %lld doubles of face traces, capacity %lld "
                      "(nx*ny*16*(k+1) must not exceed it)",
                      need, kTraceCapacity);
        message(errbuf, errbuf_len, text);
        return DGH_ERR_INVALID;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        message(errbuf, errbuf_len, "no usable current CUDA device");
        return DGH_ERR_CUDA;
    }
    double *traces = nullptr;
    {
        // Set-up, once per device and with that device current: the device address of the
        // fixed scratch array.  A host-side use of the array's name would be a host stand-in,
        // not a device address, so kernels only ever receive this looked-up pointer.
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_trace_ptr[dev]) {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_traces);
            if (e != cudaSuccess || !p) {
                message(errbuf, errbuf_len, cudaGetErrorString(e));
                return DGH_ERR_CUDA;
            }
            g_trace_ptr[dev] = static_cast<double *>(p);
        }
        traces = g_trace_ptr[dev];
    }
    const double pi = std::acos(-1.);
    const double cs = std::cos(45. * pi / 180.), sn = std::sin(45. * pi / 180.);
    const double lx = testcase == DGH_TEST_DIAGONAL ? 2. / cs : 2., ly = testcase == DGH_TEST_DIAGONAL ? 2. / sn : 2.;
    Grid g{};
    g.nx = nx;
    g.ny = ny;
    g.cells = nx * ny;
    g.hx = lx / nx;
    g.hy = ly / ny;
    g.gamma = 3.;
    Basis1D b{};
    basis_fixed(n, b);
    const double inv_step = 1. / step_size;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaSuccess;
    switch (n) {
        case 1: e = launch<1>(g, b, inv_step, u, old, speeds, r, traces, st); break;
        case 2: e = launch<2>(g, b, inv_step, u, old, speeds, r, traces, st); break;
        case 3: e = launch<3>(g, b, inv_step, u, old, speeds, r, traces, st); break;
        case 4: e = launch<4>(g, b, inv_step, u, old, speeds, r, traces, st); break;
        case 5: e = launch<5>(g, b, inv_step, u, old, speeds, r, traces, st); break;
        case 6: e = launch<6>(g, b, inv_step, u, old, speeds, r, traces, st); break;
        case 7: e = launch<7>(g, b, inv_step, u, old, speeds, r, traces, st); break;
        case 8: e = launch<8>(g, b, inv_step, u, old, speeds, r, traces, st); break;
        default: e = launch<9>(g, b, inv_step, u, old, speeds, r, traces, st); break;
    }
    if (e != cudaSuccess) {
        message(errbuf, errbuf_len, cudaGetErrorString(e));
        return DGH_ERR_CUDA;
    }
    return DGH_OK;
}
