// noalloc.cu — the sampler for callers that cannot allocate device memory.
//
// ksim_component_sample_device keeps the chunk directory that drives the
// shared-memory staging ring in a buffer the library allocates with
// cudaMalloc on the first call for each staging slot size.  Some callers
// cannot allow that: code whose device memory is owned by another allocator
// (a framework's caching pool, a serving process that pre-reserves all of
// HBM), code that must not take the implicit device synchronisation a
// cudaMalloc / cudaFree can cause inside a latency-critical loop, or an
// embedding that forbids new allocations after start-up.
// ksim_component_sample_device_noalloc serves them: its scratch is one
// file-scope __device__ array of fixed size, loaded with the library, so the
// call itself allocates nothing.
//
// The scratch holds the chunk directory, at most NOALLOC_MAX_CHUNKS records;
// components that need more are rejected with KSIM_ERR_UNSUPPORTED.  Each
// call builds the directory on the host (on the stack) and hands it to a
// one-CTA kernel as a by-value kernel parameter; that kernel writes it into
// the array and the sampling kernel follows on the same stream.  No host
// buffer is copied, so the call never waits for the stream.  The kernels'
// KSIM_FLAG_* bits go to the component's own status word (allocated when the
// component was created), read with ksim_component_status like those of every
// other sampling call.  Every call shares the array and leaves its directory
// behind: calls on one stream follow each other correctly, while calls that
// overlap on the GPU (different streams, or different host threads) race on
// it and must not be issued.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/ksim_b200.h"
#include "kernels.h"
#include "runtime.h"
#include "sample_tile.cuh"

namespace ksim {
namespace {

constexpr int NOALLOC_MAX_CHUNKS = 1024;
constexpr size_t NOALLOC_SCRATCH_BYTES = NOALLOC_MAX_CHUNKS * sizeof(ChunkDir);
constexpr int NOALLOC_MAX_DEVICES = 64;

static_assert(KSIM_NOALLOC_SCRATCH_BYTES == NOALLOC_SCRATCH_BYTES, "header and scratch size disagree");
static_assert(KSIM_NOALLOC_MAX_CHUNKS == NOALLOC_MAX_CHUNKS, "header and chunk limit disagree");

// One copy per GPU that loads the library, held until the process exits.
__device__ __align__(256) uint8_t g_sample_scratch[NOALLOC_SCRATCH_BYTES];

// Device address of g_sample_scratch per device (host code must not use the
// symbol itself: on the host it names a stand-in, not device memory).
std::mutex g_scratch_mu;
uint8_t *g_scratch_addr[NOALLOC_MAX_DEVICES] = {};

// The chunk directory as a kernel parameter: 16 bytes per chunk (term-stream
// offset, bytes, graph, term count with the end-of-graph flag in bit 31).
struct DirParam {
    int32_t n, pad[3];
    uint4 rec[NOALLOC_MAX_CHUNKS];
};
static_assert(sizeof(DirParam) <= 32764, "kernel parameters are limited to 32,764 bytes");

__global__ void __launch_bounds__(256) k_noalloc_dir(const __grid_constant__ DirParam d)
{
    ChunkDir *out = (ChunkDir *)g_sample_scratch;
    for (int i = threadIdx.x; i < d.n; i += blockDim.x) {
        const uint4 r = d.rec[i];
        ChunkDir c;
        c.off = (int64_t)r.x;
        c.bytes = (int32_t)r.y;
        c.graph = (int32_t)r.z;
        c.n_terms = (int32_t)(r.w & 0x7FFFFFFFu);
        c.end_of_graph = (int32_t)(r.w >> 31);
        c.pad0 = 0;
        c.pad1 = 0;
        out[i] = c;
    }
}

template <int W, bool STAGED>
__global__ void __launch_bounds__(256, KSIM_SAMPLE_MIN_CTAS) k_sample_noalloc(const SampleJob j)
{
    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t *bar = (uint64_t *)smem;
    uint8_t *slots = smem + BAR_BYTES;
    if (STAGED) ring_init(bar);
    uint32_t g = 0;
    constexpr int S = shots_per_thread(W);
    uint8_t *scratch = STAGED ? slots + (size_t)NSLOT * j.slot_bytes : slots;
    sample_tile<W, STAGED, false, S>(j, (int64_t)blockIdx.x * blockDim.x * S, bar, slots, g, scratch);
}

// Set-up, once per device, with that device current.
ksim_status scratch_address(int dev, uint8_t **out)
{
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES)
        return fail(KSIM_ERR_UNSUPPORTED, "device index " + std::to_string(dev) + " is beyond the " +
                                              std::to_string(NOALLOC_MAX_DEVICES) + " this entry point tracks");
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_sample_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(sample scratch)");
        g_scratch_addr[dev] = (uint8_t *)p;
    }
    *out = g_scratch_addr[dev];
    return KSIM_OK;
}

// The chunk directory of `img` for a staging slot, packed into `out`: returns
// the count, -1 if a term exceeds the slot, -2 if more than `cap` chunks are
// needed.  Same chunking rule as make_chunks (image.cpp).
int chunks_into(const HostImage &img, int64_t slot_bytes, uint4 *out, int cap)
{
    int n = 0;
    for (int k = 0; k < img.n_graphs; ++k) {
        const std::vector<int64_t> &to = img.term_off[k];
        const int G = (int)to.size() - 1;
        if (G <= 0) {
            if (n == cap) return -2;
            out[n++] = make_uint4((uint32_t)img.gdir[k].stream_off, 0u, (uint32_t)k, 0x80000000u);
            continue;
        }
        for (int t = 0; t < G;) {
            const int64_t off = to[t];
            int u = t;
            while (u < G && to[u + 1] - off <= slot_bytes) ++u;
            if (u == t) return -1;
            if (n == cap) return -2;
            out[n++] = make_uint4((uint32_t)off, (uint32_t)(to[u] - off), (uint32_t)k,
                                  (uint32_t)(u - t) | (u == G ? 0x80000000u : 0u));
            t = u;
        }
    }
    return n;
}

template <int W>
cudaError_t launch_noalloc_w(const SampleJob &j, const LaunchCfg &cfg, cudaStream_t st)
{
    const int64_t tile = (int64_t)cfg.threads * shots_per_thread(W);
    const int64_t blocks = (j.B + tile - 1) / tile;
    if (blocks > 0x7FFFFFFF) return cudaErrorInvalidConfiguration;
    const size_t smem = sample_smem_bytes(j.slot_bytes, cfg.staged != 0, W, cfg.threads);
    if (cfg.staged) {
        cudaError_t e = cudaFuncSetAttribute(k_sample_noalloc<W, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        k_sample_noalloc<W, true><<<(unsigned)blocks, cfg.threads, smem, st>>>(j);
    } else {
        cudaError_t e = cudaFuncSetAttribute(k_sample_noalloc<W, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        k_sample_noalloc<W, false><<<(unsigned)blocks, cfg.threads, smem, st>>>(j);
    }
    return cudaGetLastError();
}

cudaError_t launch_noalloc(const SampleJob &j, int W, const LaunchCfg &cfg, cudaStream_t st)
{
    switch (W) {
    case 1: return launch_noalloc_w<1>(j, cfg, st);
    case 2: return launch_noalloc_w<2>(j, cfg, st);
    case 3: return launch_noalloc_w<3>(j, cfg, st);
    case 4: return launch_noalloc_w<4>(j, cfg, st);
    case 5: return launch_noalloc_w<5>(j, cfg, st);
    case 6: return launch_noalloc_w<6>(j, cfg, st);
    case 8: return launch_noalloc_w<8>(j, cfg, st);
    case 10: return launch_noalloc_w<10>(j, cfg, st);
    case 12: return launch_noalloc_w<12>(j, cfg, st);
    case 16: return launch_noalloc_w<16>(j, cfg, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace
}  // namespace ksim

using namespace ksim;

extern "C" ksim_status ksim_component_sample_device_noalloc(ksim_component *c, const uint8_t *d_f_sel, int64_t B,
                                                            int64_t shot_offset, uint64_t seed, int32_t rng_mode,
                                                            uint8_t *d_out, int64_t out_stride, int64_t out_col0,
                                                            double *d_amp, void *stream)
{
    if (!c) return fail(KSIM_ERR_INVALID_ARGUMENT, "component is NULL");
    if (B < 0 || shot_offset < 0) return fail(KSIM_ERR_INVALID_ARGUMENT, "B and shot_offset must be >= 0");
    if (rng_mode != KSIM_RNG_XORSHIFT && rng_mode != KSIM_RNG_PHILOX)
        return fail(KSIM_ERR_INVALID_ARGUMENT, "rng_mode must be KSIM_RNG_XORSHIFT or KSIM_RNG_PHILOX");
    if (B == 0 || (c->img.n_out == 0 && !d_amp)) return KSIM_OK;
    if ((c->img.F > 0 && !d_f_sel) || (c->img.n_out > 0 && !d_out))
        return fail(KSIM_ERR_INVALID_ARGUMENT, "input or output pointer is NULL");
    if (out_col0 < 0 || out_stride < out_col0 + c->img.n_out)
        return fail(KSIM_ERR_INVALID_ARGUMENT, "out_stride must be >= out_col0 + n_out");
    if (c->image_bytes > 0xFFFFFFFFull)
        return fail(KSIM_ERR_UNSUPPORTED, "program images above 4 GiB are beyond the fixed scratch's directory "
                                          "records; use ksim_component_sample_device");
    DeviceGuard g(c->device);
    if (!g.ok) return fail(KSIM_ERR_CUDA, "cannot select the component's device");
    LaunchCfg cfg;
    int64_t wait_limit;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        cfg = c->cfg;
        wait_limit = c->wait_limit;
    }
    // the directory is built on the stack (no heap either) and travels as the
    // parameter of the kernel that writes it into the scratch
    DirParam dir;
    const int64_t chunk_slot = cfg.staged ? cfg.slot_bytes : (int64_t)1 << 30;
    const int n = chunks_into(c->img, chunk_slot, dir.rec, NOALLOC_MAX_CHUNKS);
    if (n == -1)
        return fail(KSIM_ERR_INVALID_ARGUMENT, "a term record is larger than the staging slot");
    if (n == -2)
        return fail(KSIM_ERR_UNSUPPORTED, "the component needs more than " + std::to_string(NOALLOC_MAX_CHUNKS) +
                                              " staging chunks, the most the fixed scratch of "
                                              "ksim_component_sample_device_noalloc holds; use "
                                              "ksim_component_sample_device or a larger slot_bytes");
    dir.n = n;
    dir.pad[0] = dir.pad[1] = dir.pad[2] = 0;
    uint8_t *scratch = nullptr;
    ksim_status s = scratch_address(c->device, &scratch);
    if (s != KSIM_OK) return s;
    cudaStream_t st = (cudaStream_t)stream;
    k_noalloc_dir<<<1, 256, 0, st>>>(dir);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "chunk directory kernel launch (no-alloc)");

    SampleJob j = {};
    j.image = c->d_image;
    j.gdir = (const GraphDir *)c->d_image;
    j.cdir = (const ChunkDir *)scratch;
    j.n_chunks = n;
    j.n_graphs = c->img.n_graphs;
    j.F = c->img.F;
    j.n_out = c->img.n_out;
    j.slot_bytes = cfg.staged ? cfg.slot_bytes : (int)std::max<int64_t>(c->img.max_term_bytes, 16);
    j.rng_mode = rng_mode;
    j.f = d_f_sel;
    j.f_stride = c->img.F;
    j.f_sel = nullptr;
    j.out = d_out;
    j.out_stride = out_stride;
    j.out_col0 = out_col0;
    j.out_cols = nullptr;
    j.amp = d_amp;
    j.B = B;
    j.shot_offset = shot_offset;
    j.seed = seed;
    j.status = c->d_status;
    j.wait_limit = wait_limit;
    e = launch_noalloc(j, c->img.W, cfg, st);
    if (e != cudaSuccess) return cuda_fail(e, "sample kernel launch (no-alloc)");
    return KSIM_OK;
}
