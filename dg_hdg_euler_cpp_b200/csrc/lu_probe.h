// Per-phase cycle counters for the left-looking LU (k_lu_left in dgh_kernels_lu2.cuh), force-
// included into a separate build of the library (`make probe` -> lib/libdgh_gpu_probe.so); the
// library build leaves the hooks empty.  Thread 0 of every CTA reads clock64() at each hook and
// adds the cycles since the previous hook to the phase that hook opened, in registers; the
// totals go to a per-CTA table at kernel exit.  ll_probe_reset / ll_probe_read clear and fetch
// the table ([1024 CTAs][8 phases], CTA index modulo 1024).  The counters see one warp's view
// (barrier waits included), so they split time between phases but do not measure throughput.
#pragma once
#include <cuda_runtime.h>

__device__ unsigned long long g_ll_probe[1024 * 8];

#define LL_PROBE_DECL                                                                      \
    unsigned long long llp_a0 = 0, llp_a1 = 0, llp_a2 = 0, llp_a3 = 0, llp_a4 = 0, llp_a5 = 0, \
                       llp_a6 = 0, llp_a7 = 0, llp_last = clock64();                          \
    int llp_prev = 5;
#define LL_PROBE(phase)                                                                    \
    do {                                                                                   \
        if (threadIdx.x == 0) {                                                            \
            const unsigned long long llp_t = clock64(), llp_d = llp_t - llp_last;          \
            switch (llp_prev) {                                                            \
                case 0: llp_a0 += llp_d; break;                                            \
                case 1: llp_a1 += llp_d; break;                                            \
                case 2: llp_a2 += llp_d; break;                                            \
                case 3: llp_a3 += llp_d; break;                                            \
                case 4: llp_a4 += llp_d; break;                                            \
                case 5: llp_a5 += llp_d; break;                                            \
                case 6: llp_a6 += llp_d; break;                                            \
                default: llp_a7 += llp_d; break;                                           \
            }                                                                              \
            llp_last = llp_t;                                                              \
            llp_prev = (phase);                                                            \
        }                                                                                  \
    } while (0)
#define LL_PROBE_FLUSH                                                                     \
    do {                                                                                   \
        if (threadIdx.x == 0) {                                                            \
            unsigned long long *llp_g = g_ll_probe + (blockIdx.x & 1023) * 8;              \
            llp_g[0] += llp_a0; llp_g[1] += llp_a1; llp_g[2] += llp_a2; llp_g[3] += llp_a3; \
            llp_g[4] += llp_a4; llp_g[5] += llp_a5; llp_g[6] += llp_a6; llp_g[7] += llp_a7; \
        }                                                                                  \
    } while (0)

extern "C" int ll_probe_reset() {
    static const unsigned long long zero[1024 * 8] = {};
    if (cudaDeviceSynchronize() != cudaSuccess) return 1;
    return cudaMemcpyToSymbol(g_ll_probe, zero, sizeof(zero)) == cudaSuccess ? 0 : 1;
}
extern "C" int ll_probe_read(unsigned long long *out) {
    if (cudaDeviceSynchronize() != cudaSuccess) return 1;
    return cudaMemcpyFromSymbol(out, g_ll_probe, sizeof(g_ll_probe)) == cudaSuccess ? 0 : 1;
}
