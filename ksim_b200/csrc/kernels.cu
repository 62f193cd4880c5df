// kernels.cu — sm_100a sampling and evaluation kernels.
//
// k_sample: one thread per shot runs the whole autoregressive loop of
// kokkos_sim.cpp:214-230 for its shot.  All shots of a CTA walk the same
// graphs in the same order, so the term tables are uniform across the CTA:
// they are streamed chunk by chunk (whole terms, <= slot bytes) from HBM into
// a two-slot shared-memory ring with TMA bulk copies (cp.async.bulk +
// mbarrier complete_tx), the next chunk in flight while the current one is
// evaluated; every warp then reads each column record with a broadcast
// 16-byte shared load.  The shot's parameter vector [f | m | trying] lives in
// W 64-bit registers and a parity is AND + popcount.  Waits on the mbarriers
// are bounded; a wait that runs out raises KSIM_FLAG_WAIT_TIMEOUT and the CTA
// returns after draining its copies (with a bound again).
//
// k_eval: one thread per explicit parameter row, the debug / precision entry
// of kokkos_sim.cpp:157-185 (and the per-term numerator dump).
#include <cuda_runtime.h>

#include "../../include/ksim_b200.h"
#include "kernels.h"
#include "zring.cuh"

namespace ksim {

namespace {

constexpr int NSLOT = 2;
constexpr int BAR_BYTES = 128;
constexpr long long WAIT_LIMIT = 1ll << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tma_bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    const uint32_t a = smem_u32(bar);
    for (long long it = 0; it < WAIT_LIMIT; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ double dsqrt(double x) { return __dsqrt_rn(x); }

// Bit access by position with masks only (an indexed form would move the
// register array to local memory).
template <int W>
__device__ __forceinline__ void set_bit(uint64_t (&v)[W], int pos, uint32_t bit)
{
#pragma unroll
    for (int w = 0; w < W; ++w) v[w] |= bit_range(w, pos, pos + (int)bit);
}

template <int W>
__device__ __forceinline__ uint32_t get_bit(const uint64_t (&v)[W], int pos)
{
    uint64_t x = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) x |= v[w] & bit_range(w, pos, pos + 1);
    return x != 0 ? 1u : 0u;
}

// Parameter vector of graph k: [f | m_0..m_{nm-1}] and, for k >= 1, the
// "trying" bit on every position from F+nm up to the graph's P
// (kokkos_sim.cpp:10-14 / zx_eval.hpp:86-90).
template <int W>
__device__ __forceinline__ void graph_vector(uint64_t (&vk)[W], const uint64_t (&v)[W], int F, int k,
                                             int P)
{
    const int nm = k > 0 ? k - 1 : 0;
    const int64_t lo = (int64_t)F + nm;
#pragma unroll
    for (int w = 0; w < W; ++w)
        vk[w] = (v[w] & bit_range(w, 0, lo)) | (k > 0 ? bit_range(w, lo, P) : 0ull);
}

__device__ __forceinline__ void issue_chunk(const SampleJob &j, int c, uint64_t *bar, uint8_t *slots)
{
    const ChunkDir d = j.cdir[c];
    const int slot = c & (NSLOT - 1);
    if (d.bytes > 0) {
        mbar_arrive_expect_tx(&bar[slot], (uint32_t)d.bytes);
        tma_bulk_g2s(slots + (size_t)slot * j.slot_bytes, j.image + d.off, (uint32_t)d.bytes, &bar[slot]);
    } else {
        mbar_arrive(&bar[slot]);
    }
}

template <int W, bool STAGED>
__global__ void __launch_bounds__(256) k_sample(const SampleJob j)
{
    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t *bar = (uint64_t *)smem;
    uint8_t *slots = smem + BAR_BYTES;
    const int tid = threadIdx.x;
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + tid;
    const bool act = s < j.B;

    uint64_t v[W];
#pragma unroll
    for (int w = 0; w < W; ++w) v[w] = 0;
    if (act) {
        const uint8_t *row = j.f + s * j.f_stride;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            const int lim = min(64, j.F - 64 * w);
            uint64_t x = 0;
            for (int b = 0; b < lim; ++b) {
                const int c = 64 * w + b;
                const int col = j.f_sel ? j.f_sel[c] : c;
                x |= (uint64_t)(row[col] & 1u) << b;
            }
            v[w] = x;
        }
    }
    uint64_t vk[W];
    graph_vector<W>(vk, v, j.F, 0, j.gdir[0].P);
    const uint64_t shot = (uint64_t)(j.shot_offset + s);
    uint64_t rng = xorshift_init(j.seed, shot);
    double prev = 0.0, sre = 0.0, sim = 0.0;
    uint32_t flags = 0, risk = 0;

    if (STAGED) {
        if (tid == 0) {
            mbar_init(&bar[0], 1);
            mbar_init(&bar[1], 1);
            mbar_fence_init();
        }
        __syncthreads();
        if (tid == 0)
            for (int c = 0; c < NSLOT && c < j.n_chunks; ++c) issue_chunk(j, c, bar, slots);
    }

    for (int c = 0; c < j.n_chunks; ++c) {
        const ChunkDir d = j.cdir[c];
        const uint8_t *p;
        if (STAGED) {
            const int slot = c & (NSLOT - 1);
            const bool ok = mbar_wait(&bar[slot], (uint32_t)(c / NSLOT) & 1u);
            if (__syncthreads_or(!ok)) {
                if (tid == 0) {
                    atomicOr(j.status, (uint32_t)KSIM_FLAG_WAIT_TIMEOUT);
                    // drain this copy and the one issued after it before leaving
                    mbar_wait(&bar[slot], (uint32_t)(c / NSLOT) & 1u);
                    if (c + 1 < j.n_chunks)
                        mbar_wait(&bar[(c + 1) & (NSLOT - 1)], (uint32_t)((c + 1) / NSLOT) & 1u);
                }
                return;
            }
            p = slots + (size_t)slot * j.slot_bytes;
        } else {
            p = j.image + d.off;
        }
        if (act) eval_terms<W>(p, (uint32_t)d.n_terms, vk, sre, sim, risk);
        if (d.end_of_graph) {
            const int k = d.graph;
            if (act) {
                const double mag = dsqrt(dadd(dmul(sre, sre), dmul(sim, sim)));
                if (j.amp) j.amp[s * (int64_t)(j.n_out + 1) + k] = mag;
                if (k == 0) {
                    prev = mag;
                } else {
                    const int i = k - 1;
                    const double u = j.rng_mode == KSIM_RNG_PHILOX ? philox_uniform(j.seed, shot, (uint32_t)i)
                                                                   : xorshift_uniform(rng);
                    const double ratio = __ddiv_rn(mag, prev);
                    const uint32_t bit = u < ratio ? 1u : 0u;
                    if (!(prev > 0.0)) flags |= KSIM_FLAG_PREV_NONPOSITIVE;
                    if (ratio != ratio) flags |= KSIM_FLAG_NAN;
                    set_bit<W>(v, j.F + i, bit);
                    prev = bit ? mag : dsub(prev, mag);
                }
            }
            sre = 0.0;
            sim = 0.0;
            if (k + 1 < j.n_graphs) graph_vector<W>(vk, v, j.F, k + 1, j.gdir[k + 1].P);
        }
        if (STAGED) {
            __syncthreads();
            if (tid == 0 && c + NSLOT < j.n_chunks) issue_chunk(j, c + NSLOT, bar, slots);
        }
    }

    if (act) {
        uint8_t *orow = j.out + s * j.out_stride;
        for (int i = 0; i < j.n_out; ++i) {
            const int64_t col = j.out_cols ? (int64_t)j.out_cols[i] : j.out_col0 + i;
            orow[col] = (uint8_t)get_bit<W>(v, j.F + i);
        }
        const uint32_t st = flags | (risk ? (uint32_t)KSIM_FLAG_INT64_RISK : 0u);
        if (st) atomicOr(j.status, st);
    }
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
    const GraphDir gd = j.gdir[j.graph];
    const uint8_t *p = j.image + gd.stream_off;
    uint32_t risk = 0;
    if (j.mode == EVAL_TERMS) {
        int64_t *o = (int64_t *)j.out + s * (int64_t)gd.G * 5;
        for (int t = 0; t < gd.G; ++t) {
            const TermHdr h = load_hdr(p);
            TermOut r;
            p = (h.flags & TF_SLOW) ? eval_term_exact<W>(p, h, v, r) : eval_term_fast<W>(p, h, v, r);
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
    const int64_t blocks = (j.B + threads - 1) / threads;
    if (blocks > 0x7FFFFFFF) return cudaErrorInvalidConfiguration;
    if (cfg.staged) {
        const size_t smem = staged_smem_bytes(j.slot_bytes);
        cudaError_t e = cudaFuncSetAttribute(k_sample<W, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        k_sample<W, true><<<(unsigned)blocks, threads, smem, st>>>(j);
    } else {
        k_sample<W, false><<<(unsigned)blocks, threads, 0, st>>>(j);
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

}  // namespace

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
