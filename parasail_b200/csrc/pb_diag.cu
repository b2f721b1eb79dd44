/*
 * pb_diag.cu -- diagnostics used by the benchmark: counts of this library's
 * kernel launches, the device time of the last Smith-Waterman score kernel,
 * and a microbenchmark of the DPX int16x2 add-max pipe that serves as the
 * roofline denominator of the dynamic-programming kernels.
 */
#include <cstdint>
#include <atomic>
#include <cuda_runtime.h>

#include "pb_cuda.h"

static std::atomic<long> g_launches{0};
static double g_sw16_ms = 0.0;
static std::atomic<long> g_sw16_launches{0};

extern "C" void pb_diag_count_launch(long n) { g_launches += n; }
extern "C" void pb_diag_sw16_time(double ms) { g_sw16_ms += ms; g_sw16_launches += 1; }

extern "C" long parasail_b200_kernel_launches(void) { return g_launches.load(); }
extern "C" double parasail_b200_sw16_kernel_ms(long *launches)
{
    if (launches) *launches = g_sw16_launches.load();
    return g_sw16_ms;
}
extern "C" void parasail_b200_reset_counters(void)
{
    g_launches = 0;
    g_sw16_ms = 0.0;
    g_sw16_launches = 0;
}

namespace {

/* 8 independent dependency chains of viaddmax per thread, ITERS deep */
template <int ITERS>
__global__ void k_dpx_peak(uint32_t *out, uint32_t seed)
{
    uint32_t a0 = seed ^ threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3;
    uint32_t a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
    const uint32_t g = 0xfffefffeu, c = 0x00030003u;
#pragma unroll 16
    for (int i = 0; i < ITERS; ++i) {
        a0 = __viaddmax_s16x2(a0, g, c); a1 = __viaddmax_s16x2(a1, g, c);
        a2 = __viaddmax_s16x2(a2, g, c); a3 = __viaddmax_s16x2(a3, g, c);
        a4 = __viaddmax_s16x2(a4, g, c); a5 = __viaddmax_s16x2(a5, g, c);
        a6 = __viaddmax_s16x2(a6, g, c); a7 = __viaddmax_s16x2(a7, g, c);
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = a0 ^ a1 ^ a2 ^ a3 ^ a4 ^ a5 ^ a6 ^ a7;
}

}  // namespace

/* Lane-operations per second of the int16x2 add-max pipe (one viaddmax on
 * int16x2 = 2 lane-operations), best of 5 timed launches. */
extern "C" double parasail_b200_dpx_peak(void)
{
    if (pb_cuda_init() != 0) return -1.0;
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int threads = 512, blocks = nsm * 4;
    constexpr int ITERS = 4096;
    uint32_t *out = nullptr;
    cudaMalloc(&out, sizeof(uint32_t) * threads * blocks);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_dpx_peak<ITERS><<<blocks, threads>>>(out, 1);
    float best = 1e30f;
    for (int r = 0; r < 5; ++r) {
        cudaEventRecord(e0);
        k_dpx_peak<ITERS><<<blocks, threads>>>(out, 2 + r);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        best = ms < best ? ms : best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    const double ops = 2.0 * 8.0 * ITERS * (double)threads * blocks;
    return ops / (best * 1e-3);
}
