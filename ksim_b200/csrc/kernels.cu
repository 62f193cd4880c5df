// kernels.cu — sm_100a plain sampling and evaluation kernels.
//
// k_sample: one component per launch, one CTA per tile of blockDim.x shots,
// running sample_tile (sample_tile.cuh): the autoregressive loop of
// kokkos_sim.cpp:214-230 with the term tables staged through shared memory
// by TMA bulk copies.
//
// k_eval: one thread per explicit parameter row, the debug / precision entry
// of kokkos_sim.cpp:157-185 (and the per-term numerator dump).
#include <cuda_runtime.h>

#include "../../include/ksim_b200.h"
#include "kernels.h"
#include "sample_tile.cuh"
#include "zring.cuh"

namespace ksim {

namespace {

// The kernels without the exact and 64-bit paths fit 96 registers: with
// 128-thread CTAs and 12 KiB staging slots, five CTAs per SM.  The general
// kernel keeps the two-of-256 budget.
#define KSIM_SAMPLE_BOUNDS(P) __maxnreg__((P) != PATHS_ALL ? 96 : 65536 / (256 * KSIM_SAMPLE_MIN_CTAS))
template <int W, bool STAGED, int PATHS = PATHS_ALL>
__global__ void KSIM_SAMPLE_BOUNDS(PATHS) k_sample(const SampleJob j)
{
    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t *bar = (uint64_t *)smem;
    uint8_t *slots = smem + BAR_BYTES;
    if (STAGED) ring_init(bar);
    uint32_t g = 0;
    constexpr int S = shots_per_thread(W);
    uint8_t *scratch = STAGED ? slots + (size_t)NSLOT * j.slot_bytes : slots;
    sample_tile<W, STAGED, false, S, PATHS>(j, (int64_t)blockIdx.x * blockDim.x * S, bar, slots, g,
                                                   scratch);
}

template <int W>
__global__ void __launch_bounds__(128) k_eval(const EvalJob j)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= j.B) return;
    uint64_t v[W];
    const uint8_t *row = j.params + s * j.P;
#pragma unroll
    for (int w = 0; w < W; ++w) {
        const int64_t lim = j.P - 64 * w < 64 ? j.P - 64 * w : 64;
        uint64_t x = 0;
        for (int b = 0; b < lim; ++b) x |= (uint64_t)(row[64 * w + b] & 1u) << b;
        v[w] = x;
    }
    set_one_bit<W>(v);
    const GraphDir gd = j.gdir[j.graph];
    const uint8_t *p = j.image + gd.stream_off;
    uint32_t risk = 0;
    if (j.mode == EVAL_TERMS) {
        int64_t *o = (int64_t *)j.out + s * (int64_t)gd.G * 5;
        for (int t = 0; t < gd.G; ++t) {
            const TermHdr h = load_hdr(p);
            TermOut r;
            p = eval_term<W>(p, h, v, r);
            o[5 * t + 0] = (int64_t)r.z.a;
            o[5 * t + 1] = (int64_t)r.z.b;
            o[5 * t + 2] = (int64_t)r.z.c;
            o[5 * t + 3] = (int64_t)r.z.d;
            o[5 * t + 4] = r.pw;
            risk |= r.risk;
        }
    } else {
        double re = 0.0, im = 0.0;
        eval_terms<W>(p, (uint32_t)gd.G, v, re, im, risk);
        double *o = (double *)j.out;
        if (j.mode == EVAL_ABS) {
            o[s] = dsqrt(dadd(dmul(re, re), dmul(im, im)));
        } else {
            o[2 * s] = re;
            o[2 * s + 1] = im;
        }
    }
    if (risk) atomicOr(j.status, (uint32_t)KSIM_FLAG_INT64_RISK);
}

template <int W>
cudaError_t launch_sample_w(const SampleJob &j, const LaunchCfg &cfg, cudaStream_t st)
{
    const int threads = cfg.threads;
    const int64_t tile = (int64_t)threads * shots_per_thread(W);
    const int64_t blocks = (j.B + tile - 1) / tile;
    if (blocks > 0x7FFFFFFF) return cudaErrorInvalidConfiguration;
    const size_t smem = sample_smem_bytes(j.slot_bytes, cfg.staged != 0, W, threads);
    if (cfg.staged && cfg.paths == PATHS_NARROW && W <= 4) {
        cudaError_t e = cudaFuncSetAttribute(k_sample<W, true, PATHS_NARROW>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        k_sample<W, true, PATHS_NARROW><<<(unsigned)blocks, threads, smem, st>>>(j);
    } else if (cfg.staged && cfg.paths == PATHS_NARROW_HYBRID && W <= 4) {
        cudaError_t e = cudaFuncSetAttribute(k_sample<W, true, PATHS_NARROW_HYBRID>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        k_sample<W, true, PATHS_NARROW_HYBRID><<<(unsigned)blocks, threads, smem, st>>>(j);
    } else if (cfg.staged) {
        cudaError_t e = cudaFuncSetAttribute(k_sample<W, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        k_sample<W, true><<<(unsigned)blocks, threads, smem, st>>>(j);
    } else {
        cudaError_t e = cudaFuncSetAttribute(k_sample<W, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        k_sample<W, false><<<(unsigned)blocks, threads, smem, st>>>(j);
    }
    return cudaGetLastError();
}

template <int W>
cudaError_t launch_eval_w(const EvalJob &j, cudaStream_t st)
{
    const int threads = 128;
    const int64_t blocks = (j.B + threads - 1) / threads;
    if (blocks > 0x7FFFFFFF) return cudaErrorInvalidConfiguration;
    k_eval<W><<<(unsigned)blocks, threads, 0, st>>>(j);
    return cudaGetLastError();
}

// One output byte per thread (grid-stride): HBM-bound byte work.
__global__ void __launch_bounds__(256) k_unpack_bits(const uint8_t *__restrict__ packed, int64_t rows,
                                                     int64_t packed_row, int64_t n_cols, uint8_t *__restrict__ out)
{
    const int64_t n = rows * n_cols;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = i / n_cols, c = i - r * n_cols;
        out[i] = (packed[r * packed_row + (c >> 3)] >> (c & 7)) & 1u;
    }
}

// One packed byte per thread (grid-stride).
__global__ void __launch_bounds__(256) k_pack_bits(const uint8_t *__restrict__ bytes, int64_t rows, int64_t n_cols,
                                                   int64_t packed_row, uint8_t *__restrict__ out)
{
    const int64_t n = rows * packed_row;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = i / packed_row, b = i - r * packed_row;
        const uint8_t *src = bytes + r * n_cols + 8 * b;
        const int64_t m = n_cols - 8 * b < 8 ? n_cols - 8 * b : 8;
        uint32_t x = 0;
        for (int k = 0; k < m; ++k) x |= (uint32_t)(src[k] & 1u) << k;
        out[i] = (uint8_t)x;
    }
}

unsigned byte_grid(int64_t n)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t want = (n + 255) / 256;
    const int64_t cap = (int64_t)sms * 8;
    return (unsigned)(want < cap ? (want > 0 ? want : 1) : cap);
}

}  // namespace

cudaError_t launch_unpack_bits(const uint8_t *packed, int64_t rows, int64_t packed_row, int64_t n_cols, uint8_t *out,
                               cudaStream_t st)
{
    if (rows <= 0 || n_cols <= 0) return cudaSuccess;
    k_unpack_bits<<<byte_grid(rows * n_cols), 256, 0, st>>>(packed, rows, packed_row, n_cols, out);
    return cudaGetLastError();
}

cudaError_t launch_pack_bits(const uint8_t *bytes, int64_t rows, int64_t n_cols, int64_t packed_row, uint8_t *out,
                             cudaStream_t st)
{
    if (rows <= 0 || n_cols <= 0) return cudaSuccess;
    k_pack_bits<<<byte_grid(rows * packed_row), 256, 0, st>>>(bytes, rows, n_cols, packed_row, out);
    return cudaGetLastError();
}

size_t staged_smem_bytes(int slot_bytes) { return (size_t)BAR_BYTES + (size_t)NSLOT * (size_t)slot_bytes; }

cudaError_t launch_sample(const SampleJob &job, int W, const LaunchCfg &cfg, cudaStream_t st)
{
    if (job.B <= 0) return cudaSuccess;
    if (cfg.threads <= 0 || cfg.threads > 256 || (cfg.threads & 31)) return cudaErrorInvalidConfiguration;
    switch (W) {
    case 1: return launch_sample_w<1>(job, cfg, st);
    case 2: return launch_sample_w<2>(job, cfg, st);
    case 3: return launch_sample_w<3>(job, cfg, st);
    case 4: return launch_sample_w<4>(job, cfg, st);
    case 5: return launch_sample_w<5>(job, cfg, st);
    case 6: return launch_sample_w<6>(job, cfg, st);
    case 8: return launch_sample_w<8>(job, cfg, st);
    case 10: return launch_sample_w<10>(job, cfg, st);
    case 12: return launch_sample_w<12>(job, cfg, st);
    case 16: return launch_sample_w<16>(job, cfg, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_eval(const EvalJob &job, int W, cudaStream_t st)
{
    if (job.B <= 0) return cudaSuccess;
    switch (W) {
    case 1: return launch_eval_w<1>(job, st);
    case 2: return launch_eval_w<2>(job, st);
    case 3: return launch_eval_w<3>(job, st);
    case 4: return launch_eval_w<4>(job, st);
    case 5: return launch_eval_w<5>(job, st);
    case 6: return launch_eval_w<6>(job, st);
    case 8: return launch_eval_w<8>(job, st);
    case 10: return launch_eval_w<10>(job, st);
    case 12: return launch_eval_w<12>(job, st);
    case 16: return launch_eval_w<16>(job, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace ksim
