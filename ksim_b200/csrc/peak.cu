// peak.cu — integer-pipe throughput microbenchmark (roofline denominator).
//
// The sampler is bound by 32-bit integer ALU work (adds with carry, logic,
// funnel shifts, popcount), not by HBM or tensor cores.  This kernel measures
// what the SMs of the box actually sustain for that instruction mix: every
// thread runs 8 independent chains of add / xor-and / shift steps, grid sized
// to fill every SM, timed with CUDA events.  Reported as int32 lane-ops/s.
#include <cuda_runtime.h>

#include "../../include/ksim_b200.h"
#include "runtime.h"

namespace ksim {
namespace {

__global__ void __launch_bounds__(256) k_int_peak(uint32_t *sink, int iters, uint32_t seed)
{
    uint32_t a0 = threadIdx.x ^ seed, a1 = a0 * 3u, a2 = a0 * 5u, a3 = a0 * 7u;
    uint32_t a4 = a0 * 11u, a5 = a0 * 13u, a6 = a0 * 17u, a7 = a0 * 19u;
    const uint32_t k = seed | 1u;
    for (int i = 0; i < iters; ++i) {
        // 4 ops per chain per step: add, shift, and-xor (one LOP3), funnel shift
#define STEP(x) x = (x + k); x = (x & 0x5bd1e995u) ^ (x >> 3); x = __funnelshift_l(x, x, 7);
        STEP(a0) STEP(a1) STEP(a2) STEP(a3) STEP(a4) STEP(a5) STEP(a6) STEP(a7)
#undef STEP
    }
    const uint32_t r = a0 ^ a1 ^ a2 ^ a3 ^ a4 ^ a5 ^ a6 ^ a7;
    if (r == 0x12345678u) sink[blockIdx.x] = r;  // keeps the chains live
}

// The integer ALU alone: 8 independent chains of a three-input xor (one
// LOP3) and a three-input add (one IADD3) per step, no shifts, multiplies or
// popcounts.  2 ops per chain per step.
__global__ void __launch_bounds__(256) k_alu_peak(uint32_t *sink, int iters, uint32_t seed)
{
    uint32_t x[8], y[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        x[c] = (threadIdx.x + 977u * c) ^ seed;
        y[c] = x[c] * 2654435761u + c;
    }
    const uint32_t k1 = seed | 1u, k2 = seed * 3u + 7u;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            x[c] = x[c] ^ y[c] ^ k1;
            y[c] = y[c] + x[c] + k2;
        }
    }
    uint32_t r = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) r ^= x[c] ^ y[c];
    if (r == 0x12345678u) sink[blockIdx.x] = r;  // keeps the chains live
}

// Best-of-4 event time (ms) of `launch` after one warm-up run.
template <typename F>
cudaError_t time_best(F launch, float &best)
{
    cudaEvent_t t0, t1;
    cudaError_t e = cudaEventCreate(&t0);
    if (e == cudaSuccess) e = cudaEventCreate(&t1);
    if (e != cudaSuccess) return e;
    best = 1e30f;
    for (int rep = 0; rep < 5 && e == cudaSuccess; ++rep) {
        cudaEventRecord(t0);
        launch(rep);
        cudaEventRecord(t1);
        e = cudaEventSynchronize(t1);
        float m = 0;
        if (e == cudaSuccess) cudaEventElapsedTime(&m, t0, t1);
        if (rep > 0 && m < best) best = m;
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    return e;
}

}  // namespace
}  // namespace ksim

extern "C" ksim_status ksim_measure_alu_peak(int32_t device, double *ops_per_s, double *ms)
{
    using namespace ksim;
    if (!ops_per_s) return fail(KSIM_ERR_INVALID_ARGUMENT, "ops_per_s is NULL");
    DeviceGuard g(device);
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = sms * 8, threads = 256, iters = 4096;
    uint32_t *sink = nullptr;
    cudaError_t e = cudaMalloc(&sink, sizeof(uint32_t) * blocks);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(sink)");
    float best = 0;
    e = time_best([&](int rep) { k_alu_peak<<<blocks, threads>>>(sink, iters, 0x85ebca6bu + rep); }, best);
    cudaFree(sink);
    if (e != cudaSuccess) return cuda_fail(e, "alu peak kernel");
    const double ops = (double)blocks * threads * iters * 8.0 * 2.0;
    *ops_per_s = ops / (best * 1e-3);
    if (ms) *ms = best;
    return KSIM_OK;
}

extern "C" ksim_status ksim_measure_int_peak(int32_t device, double *ops_per_s, double *ms)
{
    using namespace ksim;
    if (!ops_per_s) return fail(KSIM_ERR_INVALID_ARGUMENT, "ops_per_s is NULL");
    DeviceGuard g(device);
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = sms * 8, threads = 256, iters = 4096;
    uint32_t *sink = nullptr;
    cudaError_t e = cudaMalloc(&sink, sizeof(uint32_t) * blocks);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(sink)");
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    float best = 1e30f;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(t0);
        k_int_peak<<<blocks, threads>>>(sink, iters, 0x9e3779b9u + rep);
        cudaEventRecord(t1);
        e = cudaEventSynchronize(t1);
        if (e != cudaSuccess) break;
        float m = 0;
        cudaEventElapsedTime(&m, t0, t1);
        if (rep > 0 && m < best) best = m;
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaFree(sink);
    if (e != cudaSuccess) return cuda_fail(e, "int peak kernel");
    const double ops = (double)blocks * threads * iters * 8.0 * 4.0;
    *ops_per_s = ops / (best * 1e-3);
    if (ms) *ms = best;
    return KSIM_OK;
}
