// sample_tile.cuh — the per-CTA sampling loop shared by the plain kernel
// (one component per launch) and the persistent batched kernel.
//
// One thread per shot runs the autoregressive loop of kokkos_sim.cpp:214-230:
// |A_0|, then for every output i, p1 = |A_{i+1}|, one uniform, bit = u < p1/prev,
// prev = bit ? p1 : prev - p1.  All shots of the CTA walk the same graphs in
// the same order, so the term tables are uniform across the CTA: they stream
// chunk by chunk (whole terms, <= slot bytes) from HBM into a two-slot
// shared-memory ring with TMA bulk copies (cp.async.bulk + mbarrier
// complete_tx); the copy of chunk c+2 is in flight while chunk c+1 is
// evaluated.  The shot's parameter vector [f | m | trying] is W 64-bit
// registers.
//
// Parities are computed warp-sliced.  Each warp keeps, in shared memory, one
// 64-bit ballot word per parameter bit (bit s = that bit of the warp's shot
// s; shots 0-31 are the lanes' first shots, 32-63 their second); a parity
// row is the XOR of the ballot words of its few set bits, so lane l builds
// row 32b + l of a block for all 64 shots with a handful of loads, and a
// 32x32 bit transpose over the warp (five shuffle rounds) gives every shot
// its 32 row parities as one word.  The term arithmetic then reads
// row-parity bit ranges (zring.cuh, eval_term_rows).
//
// Every mbarrier wait is bounded.  A wait that runs out raises
// KSIM_FLAG_WAIT_TIMEOUT; the CTA then waits (bounded again) for the copies it
// issued and returns false without writing outputs.
//
// CG = true reads every job-dependent array (directories, f rows, column
// maps) with L2-only loads.  The serving loop needs that: its CTAs live
// across requests, and a request's buffers may reuse memory an earlier
// request of the same kernel lifetime read through this SM's L1.
#pragma once
#include <cuda_runtime.h>

#include "../../include/ksim_b200.h"
#include "kernels.h"
#include "zring.cuh"

namespace ksim {

constexpr int NSLOT = 2;
constexpr int BAR_BYTES = 128;
static_assert(ROW_WORDS == NB_MAX + 1, "row-parity words per shot: one term's blocks and a spare");
// Polls of an mbarrier wait before it gives up (each poll is one try_wait,
// which itself suspends for a hardware-defined interval).  A job may set its
// own bound (SampleJob::wait_limit) for the waits of its chunks, counted in
// non-blocking test_wait polls 64 ns apart; the waits that drain a CTA's
// copies after a timeout always use this one.
constexpr long long WAIT_LIMIT = 1ll << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

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
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit = WAIT_LIMIT)
{
    const uint32_t a = smem_u32(bar);
    for (long long it = 0; it < limit; ++it) {
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

// A wait of at most `polls` non-blocking tests, 64 ns apart (a job's own bound).
__device__ __forceinline__ bool mbar_poll(uint64_t *bar, uint32_t parity, long long polls)
{
    const uint32_t a = smem_u32(bar);
    for (long long it = 0; it < polls; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
        __nanosleep(64);
    }
    return false;
}

// Prepare the barriers of a CTA's staging ring (once per CTA).
__device__ __forceinline__ void ring_init(uint64_t *bar)
{
    if (threadIdx.x == 0) {
        for (int i = 0; i < NSLOT; ++i) mbar_init(&bar[i], 1);
        mbar_fence_init();
    }
    __syncthreads();
}

__device__ __forceinline__ double dsqrt(double x) { return __dsqrt_rn(x); }

// Loads of job-dependent data: plain, or L2-only when CG (see above).
template <bool CG, typename T>
__device__ __forceinline__ T ldj(const T *p)
{
    if (CG) return __ldcg(p);
    return *p;
}

template <bool CG>
__device__ __forceinline__ ChunkDir ld_chunk(const ChunkDir *p)
{
    if (!CG) return *p;
    const longlong2 *q = (const longlong2 *)p;
    const longlong2 a = __ldcg(q), b = __ldcg(q + 1);
    ChunkDir d;
    d.off = a.x;
    d.bytes = (int32_t)(uint32_t)a.y;
    d.graph = (int32_t)(a.y >> 32);
    d.n_terms = (int32_t)(uint32_t)b.x;
    d.end_of_graph = (int32_t)(b.x >> 32);
    d.pad0 = (int32_t)(uint32_t)b.y;
    d.pad1 = (int32_t)(b.y >> 32);
    return d;
}

template <bool CG>
__device__ __forceinline__ int graph_params(const GraphDir *g)
{
    return CG ? __ldcg(&g->P) : g->P;
}

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

// 32x32 bit transposes across the warp: lane i holds row i (bit b = column
// b) and gets column i back (bit b = row b).  Round j swaps the off-diagonal
// j x j blocks of lane pairs (i, i ^ j): the lower lane keeps its bits with
// b & j clear and takes its partner's, shifted up by j, into the others; the
// upper lane the mirror image.  The 16- and 8-bit rounds move whole bytes,
// one byte permute each; the 4-, 2- and 1-bit rounds rotate and merge.
__device__ __forceinline__ uint32_t tr_round_bytes(uint32_t x, uint32_t y, int j, bool up)
{
    // lower: [x0 x1 y0 y1] (j = 16) or [x0 y0 x2 y2] (j = 8); upper the mirror
    const uint32_t sel = j == 16 ? (up ? 0x3276u : 0x5410u) : (up ? 0x3715u : 0x6240u);
    return __byte_perm(x, y, sel);
}

__device__ __forceinline__ void transpose32x2(uint32_t &x0, uint32_t &x1, int lane)
{
#pragma unroll
    for (int j = 16; j >= 8; j >>= 1) {
        const bool up = (lane & j) != 0;
        const uint32_t y0 = __shfl_xor_sync(~0u, x0, j);
        const uint32_t y1 = __shfl_xor_sync(~0u, x1, j);
        x0 = tr_round_bytes(x0, y0, j, up);
        x1 = tr_round_bytes(x1, y1, j, up);
    }
#pragma unroll
    for (int j = 4; j >= 1; j >>= 1) {
        const uint32_t m = j == 4 ? 0xF0F0F0F0u : j == 2 ? 0xCCCCCCCCu : 0xAAAAAAAAu;  // bits b with b & j
        const bool up = (lane & j) != 0;
        const uint32_t keep = up ? m : ~m;
        const uint32_t sh = up ? (uint32_t)j : (uint32_t)(32 - j);  // rotate right by j, or left by j
        const uint32_t y0 = __shfl_xor_sync(~0u, x0, j);
        const uint32_t y1 = __shfl_xor_sync(~0u, x1, j);
        x0 = (x0 & keep) | (__funnelshift_r(y0, y0, sh) & ~keep);
        x1 = (x1 & keep) | (__funnelshift_r(y1, y1, sh) & ~keep);
    }
}

__device__ __forceinline__ uint32_t transpose32(uint32_t x0, int lane)
{
#pragma unroll
    for (int j = 16; j >= 8; j >>= 1) {
        const uint32_t y0 = __shfl_xor_sync(~0u, x0, j);
        x0 = tr_round_bytes(x0, y0, j, (lane & j) != 0);
    }
#pragma unroll
    for (int j = 4; j >= 1; j >>= 1) {
        const uint32_t m = j == 4 ? 0xF0F0F0F0u : j == 2 ? 0xCCCCCCCCu : 0xAAAAAAAAu;
        const bool up = (lane & j) != 0;
        const uint32_t keep = up ? m : ~m;
        const uint32_t sh = up ? (uint32_t)j : (uint32_t)(32 - j);
        const uint32_t y0 = __shfl_xor_sync(~0u, x0, j);
        x0 = (x0 & keep) | (__funnelshift_r(y0, y0, sh) & ~keep);
    }
    return x0;
}

// Ballot words of parameter bits [k0, k1) (warp-uniform bounds).
template <int W, int S>
__device__ __forceinline__ void ballot_words(uint64_t *sw, const uint64_t (&vk)[S][W], int k0, int k1, int lane)
{
    for (int k = k0; k < k1; ++k) {
        uint64_t x = __ballot_sync(~0u, get_bit<W>(vk[0], k));
        if (S > 1) x |= (uint64_t)__ballot_sync(~0u, get_bit<W>(vk[S - 1], k)) << 32;
        if (lane == (k & 31)) sw[k] = x;
    }
    __syncwarp();
}

// Ballot words of positions [k0, k1) that hold the same bit for every shot
// (x = all ones or zero); the caller syncs the warp.
__device__ __forceinline__ void uniform_words(uint64_t *sw, int k0, int k1, uint64_t x, int lane)
{
    for (int k = k0 + lane; k < k1; k += 32) sw[k] = x;
}

// The exact path out of line: rare, and inlined it would take registers from
// the fast path of every term.
template <int W>
__device__ __noinline__ void eval_term_exact_call(const uint8_t *p, const TermHdr &h, const uint64_t (&v)[W],
                                                  TermOut &o)
{
    eval_term_exact<W>(p, h, v, o);
}

// Terms of one chunk for the warp's shots, adding each term's complex value
// to (sum_re[s], sum_im[s]) in order (the warp-sliced form of eval_terms_s).
// sw: the warp's ballot words; wb: this thread's row-parity words (block b,
// shot r at wb[b * S * blockDim + r * blockDim]).
// PATHS: which term paths the program uses (the host checked), so the others
// are not compiled in: PATHS_ALL, PATHS_NARROW (every term on 32-bit words),
// PATHS_NARROW_HYBRID (32-bit words and the hybrid path).
enum : int { PATHS_ALL = 0, PATHS_NARROW = 1, PATHS_NARROW_HYBRID = 2 };
template <int W, int S, int PATHS = PATHS_ALL>
__device__ __forceinline__ const uint8_t *eval_terms_warp(const uint8_t *p, uint32_t n_terms,
                                                          const uint64_t (&v)[S][W], const uint8_t *sw,
                                                          uint32_t *wb, double (&sum_re)[S], double (&sum_im)[S],
                                                          uint32_t &risk, uint32_t live, int lane)
{
    const int nt = (int)blockDim.x, wstride = S * nt;
    for (uint32_t t = 0; t < n_terms; ++t) {
        const TermHdr h = load_hdr(p);
        TermOut o[S];
        if (PATHS == PATHS_ALL && (h.flags & TF_SLOW)) {
#pragma unroll
            for (int s = 0; s < S; ++s) eval_term_exact_call<W>(p, h, v[s], o[s]);
        } else {
            RowSums sums[S];
#pragma unroll
            for (int s = 0; s < S; ++s) row_sums_init(sums[s], h);
            const uint16_t *dead_pw = term_dead_pw(p, h);
            const uint8_t *blk = p + term_blocks_off(h);
            for (uint32_t b = 0; b < h.nb; ++b) {
                const BlockHead m = load_block_head(blk);
                const uint32_t n_pairs = m.n_pairs;
                const uint32_t *ix = (const uint32_t *)(blk + BLOCK_HEAD_BYTES) + lane;
                uint64_t acc = 0;
#pragma unroll 4
                for (uint32_t i = 0; i < n_pairs; ++i) {
                    const uint32_t x = ix[32 * i];
                    acc ^= *(const uint64_t *)(sw + (x & 0xFFFFu)) ^ *(const uint64_t *)(sw + (x >> 16));
                }
                if (S > 1) {
                    uint32_t x0 = (uint32_t)acc, x1 = (uint32_t)(acc >> 32);
                    transpose32x2(x0, x1, lane);
                    wb[b * wstride] = x0;
                    wb[b * wstride + nt] = x1;
                    row_sums_add(sums[0], x0, m, b, dead_pw);
                    row_sums_add(sums[S - 1], x1, m, b, dead_pw);
                } else {
                    const uint32_t x0 = transpose32((uint32_t)acc, lane);
                    wb[b * wstride] = x0;
                    row_sums_add(sums[0], x0, m, b, dead_pw);
                }
                blk += BLOCK_HEAD_BYTES + 128 * n_pairs;
            }
            RowBits bits[S];
#pragma unroll
            for (int s = 0; s < S; ++s) {
                bits[s].w = wb + s * nt;
                bits[s].stride = wstride;
            }
            if (PATHS == PATHS_NARROW)
                eval_term_rows<uint32_t, uint32_t, S>(p, h, sums, bits, o);
            else if (PATHS == PATHS_NARROW_HYBRID) {
                if (h.flags & TF_NARROW)
                    eval_term_rows<uint32_t, uint32_t, S>(p, h, sums, bits, o);
                else
                    eval_term_rows<uint32_t, uint64_t, S>(p, h, sums, bits, o);
            } else {
                eval_term_rows_any<S>(p, h, sums, bits, o);
            }
        }
#pragma unroll
        for (int s = 0; s < S; ++s) {
            double re, im;
            term_complex(o[s], p, h.flags, re, im);
            sum_re[s] = dadd(sum_re[s], re);
            sum_im[s] = dadd(sum_im[s], im);
            risk |= o[s].risk & (live >> s);
        }
        p += h.rec_bytes;
    }
    return p;
}

// Parameter vector of graph k: [f | m_0..m_{nm-1}] and, for k >= 1, the
// "trying" bit on every position from F+nm up to the graph's P
// (kokkos_sim.cpp:10-14 / zx_eval.hpp:86-90), plus the constant-one top bit.
template <int W>
__device__ __forceinline__ void graph_vector(uint64_t (&vk)[W], const uint64_t (&v)[W], int F, int k, int P)
{
    const int nm = k > 0 ? k - 1 : 0;
    const int64_t lo = (int64_t)F + nm;
#pragma unroll
    for (int w = 0; w < W; ++w) vk[w] = (v[w] & bit_range(w, 0, lo)) | (k > 0 ? bit_range(w, lo, P) : 0ull);
    set_one_bit<W>(vk);
}

// Issue the copy of chunk c of job j; gidx is its position in the CTA's
// running chunk count (it picks the slot and the barrier phase).
template <bool CG>
__device__ __forceinline__ void issue_chunk(const SampleJob &j, int c, uint32_t gidx, uint64_t *bar, uint8_t *slots)
{
    const ChunkDir d = ld_chunk<CG>(j.cdir + c);
    const int slot = (int)(gidx & (NSLOT - 1));
    if (d.bytes > 0) {
        mbar_arrive_expect_tx(&bar[slot], (uint32_t)d.bytes);
        tma_bulk_g2s(slots + (size_t)slot * j.slot_bytes, j.image + d.off, (uint32_t)d.bytes, &bar[slot]);
    } else {
        mbar_arrive(&bar[slot]);
    }
}

// Sample shots [s0, s0 + blockDim.x) of job j.  g is the CTA's running chunk
// count (advanced by the job's chunk count).  Returns false after a wait
// timeout (the CTA must then stop using the ring).
// scratch: sliced_smem_bytes(W, blockDim.x) bytes of shared memory.
template <int W, bool STAGED, bool CG = false, int S = 1, int PATHS = PATHS_ALL>
__device__ __forceinline__ bool sample_tile(const SampleJob &j, const int64_t s0, uint64_t *bar, uint8_t *slots,
                                            uint32_t &g, uint8_t *scratch)
{
    const int tid = threadIdx.x, lane = tid & 31;
    uint64_t *sw = (uint64_t *)scratch + (size_t)(tid >> 5) * ballot_words_per_warp(W);
    uint32_t *wb = (uint32_t *)(scratch + (size_t)(blockDim.x >> 5) * ballot_words_per_warp(W) * 8) + tid;
    const int F = j.F;
    // thread tid owns shots s0 + tid + r * blockDim.x, r < S
    int64_t sh[S];
    bool act[S];
    bool any = false;
    uint32_t live = 0;
    uint64_t v[S][W];
#pragma unroll
    for (int r = 0; r < S; ++r) {
        sh[r] = s0 + tid + (int64_t)r * blockDim.x;
        act[r] = sh[r] < j.B;
        any |= act[r];
        live |= act[r] ? 1u << r : 0u;
#pragma unroll
        for (int w = 0; w < W; ++w) v[r][w] = 0;
        if (act[r]) {
            const uint8_t *row = j.f + sh[r] * j.f_stride;
#pragma unroll
            for (int w = 0; w < W; ++w) {
                const int lim = min(64, F - 64 * w);
                uint64_t x = 0;
                for (int b = 0; b < lim; ++b) {
                    const int c = 64 * w + b;
                    const int col = j.f_sel ? ldj<CG>(j.f_sel + c) : c;
                    x |= (uint64_t)(ldj<CG>(row + col) & 1u) << b;
                }
                v[r][w] = x;
            }
        }
    }
    uint64_t vk[S][W];
    int Pk = graph_params<CG>(j.gdir);
#pragma unroll
    for (int r = 0; r < S; ++r) graph_vector<W>(vk[r], v[r], F, 0, Pk);
    ballot_words<W, S>(sw, vk, 0, 64 * W, lane);
    if (lane == 0) {
        sw[64 * W] = 0;  // the zero word of short rows
        sw[64 * W + 1] = 0;
    }
    __syncwarp();
    const bool warp_any = __any_sync(~0u, any);
    uint64_t rng[S];
    double prev[S], sre[S], sim[S];
#pragma unroll
    for (int r = 0; r < S; ++r) {
        rng[r] = xorshift_init(j.seed, (uint64_t)(j.shot_offset + sh[r]));
        prev[r] = 0.0;
        sre[r] = 0.0;
        sim[r] = 0.0;
    }
    uint32_t flags = 0, risk = 0;
    const int nch = j.n_chunks;

    if (STAGED && tid == 0)
        for (int c = 0; c < NSLOT && c < nch; ++c) issue_chunk<CG>(j, c, g + (uint32_t)c, bar, slots);

    for (int c = 0; c < nch; ++c) {
        const ChunkDir d = ld_chunk<CG>(j.cdir + c);
        const uint32_t gc = g + (uint32_t)c;
        const uint8_t *p;
        if (STAGED) {
            const int slot = (int)(gc & (NSLOT - 1));
            const bool ok = j.wait_limit > 0 ? mbar_poll(&bar[slot], (gc / NSLOT) & 1u, j.wait_limit)
                                             : mbar_wait(&bar[slot], (gc / NSLOT) & 1u);
            if (__syncthreads_or(!ok)) {
                if (tid == 0) {
                    atomicOr(j.status, (uint32_t)KSIM_FLAG_WAIT_TIMEOUT);
                    mbar_wait(&bar[slot], (gc / NSLOT) & 1u);
                    if (c + 1 < nch) mbar_wait(&bar[(gc + 1) & (NSLOT - 1)], ((gc + 1) / NSLOT) & 1u);
                }
                return false;
            }
            p = slots + (size_t)slot * j.slot_bytes;
        } else {
            p = j.image + d.off;
        }
        if (warp_any) eval_terms_warp<W, S, PATHS>(p, (uint32_t)d.n_terms, vk, (const uint8_t *)sw, wb, sre, sim, risk,
                                            live, lane);
        if (d.end_of_graph) {
            const int k = d.graph;
#pragma unroll
            for (int r = 0; r < S; ++r) {
                if (!act[r]) continue;
                const double mag = dsqrt(dadd(dmul(sre[r], sre[r]), dmul(sim[r], sim[r])));
                if (j.amp) j.amp[sh[r] * (int64_t)(j.n_out + 1) + k] = mag;
                if (k == 0) {
                    prev[r] = mag;
                } else {
                    const int i = k - 1;
                    const double u = j.rng_mode == KSIM_RNG_PHILOX
                                         ? philox_uniform(j.seed, (uint64_t)(j.shot_offset + sh[r]), (uint32_t)i)
                                         : xorshift_uniform(rng[r]);
                    const double ratio = __ddiv_rn(mag, prev[r]);
                    const uint32_t bit = u < ratio ? 1u : 0u;
                    if (!(prev[r] > 0.0)) flags |= KSIM_FLAG_PREV_NONPOSITIVE;
                    if (ratio != ratio) flags |= KSIM_FLAG_NAN;
                    set_bit<W>(v[r], F + i, bit);
                    prev[r] = bit ? mag : dsub(prev[r], mag);
                }
            }
#pragma unroll
            for (int r = 0; r < S; ++r) {
                sre[r] = 0.0;
                sim[r] = 0.0;
            }
            if (k + 1 < j.n_graphs) {
                // graph k + 1's vector: [0, lo) from v, trying bits [lo, Pn)
                // = 1, zeros above (lo = F + k).  Against graph k's only the
                // output just sampled (position lo - 1, k >= 1) differs
                // between shots: it gets a ballot.  The trying bits that
                // enter ([max(lo, P_k), Pn); all of [lo, Pn) after graph 0,
                // which has none) and the positions that leave the vector
                // ([max(lo, Pn), P_k)) are the same for every shot: their
                // words are written whole.  The top bit (the constant 1)
                // stays.
                const int Pn = graph_params<CG>(j.gdir + k + 1);
#pragma unroll
                for (int r = 0; r < S; ++r) graph_vector<W>(vk[r], v[r], F, k + 1, Pn);
                const int top = 64 * W - 1, lo = F + k;
                const int on0 = k > 0 ? max(lo, Pk) : lo;
                uniform_words(sw, on0, min(Pn, top), ~0ull, lane);
                uniform_words(sw, max(lo, Pn), min(Pk, top), 0ull, lane);
                if (k > 0 && lo - 1 < top) ballot_words<W, S>(sw, vk, lo - 1, lo, lane);  // ends with a warp sync
                else __syncwarp();
                Pk = Pn;
            }
        }
        if (STAGED) {
            __syncthreads();
            if (tid == 0 && c + NSLOT < nch) issue_chunk<CG>(j, c + NSLOT, gc + NSLOT, bar, slots);
        }
    }
    g += (uint32_t)nch;

#pragma unroll
    for (int r = 0; r < S; ++r) {
        if (!act[r]) continue;
        uint8_t *orow = j.out + sh[r] * j.out_stride;
        for (int i = 0; i < j.n_out; ++i) {
            const int64_t col = j.out_cols ? (int64_t)ldj<CG>(j.out_cols + i) : j.out_col0 + i;
            orow[col] = (uint8_t)get_bit<W>(v[r], F + i);
        }
    }
    if (any) {
        const uint32_t st = flags | (risk ? (uint32_t)KSIM_FLAG_INT64_RISK : 0u);
        if (st) atomicOr(j.status, st);
    }
    return true;
}

}  // namespace ksim
