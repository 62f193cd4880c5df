// batch.cu — many components / programs in one persistent, graph-captured launch.
//
// Work is cut into items (job, tile of blockDim.x shots).  Items are ordered
// longest-first (cost = tile shots x term-stream bytes of the job's component)
// and a grid of (CTAs per SM x SMs) persistent CTAs pulls them from a device
// work counter with one atomicAdd per item, so programs with uneven term
// counts, output counts and shot counts share the GPU with little tail.  A
// CTA keeps one staging ring for its whole life; its running chunk count picks
// each copy's slot and barrier phase across items of different jobs.
//
// Jobs are dispatched on their parameter-word class at run time: one kernel
// covers W <= 4 (every workload of the benchmark), a second W in 5..16; a
// batch needing only one class is one launch.  The counter reset and the
// launch(es) are captured once into a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/ksim_b200.h"
#include "kernels.h"
#include "runtime.h"
#include "sample_tile.cuh"

namespace ksim {

struct BatchJobDev {
    SampleJob j;
    int32_t W, paths;  // paths: the component's term paths (LaunchCfg::paths)
    int64_t pad1;
};

struct BatchItem {
    int32_t job, pad;
    int64_t s0;
};

namespace {

// Class 0 runs W <= 4, class 1 the wider vectors; the parity scratch is
// sized for the largest W among a launch's jobs (smaller scratch leaves more
// of the SM's shared storage to L1).
size_t batch_smem_bytes(int slot_bytes, int max_w, int threads)
{
    return sample_smem_bytes(slot_bytes, true, max_w, threads);
}

// One item's body per (W, term paths), each out of line: register-allocated
// on its own, so the 32-bit and hybrid bodies keep the allocation of the
// plain kernels compiled for those paths, and the general body (64-bit words,
// exact path; rare) cannot raise it.  An item is a whole tile of shots, so
// the call costs nothing measurable.
// Shots per thread of an item: two for W <= 4 (one for the hybrid and
// general bodies when KSIM_BATCH_WIDE_S is 1, for a smaller register budget),
// one for wider vectors.
#ifndef KSIM_BATCH_WIDE_S
#define KSIM_BATCH_WIDE_S 2
#endif
__host__ __device__ constexpr int batch_spt(int W, int paths)
{
    return paths == PATHS_NARROW ? shots_per_thread(W) : (W <= 4 ? KSIM_BATCH_WIDE_S : 1);
}

template <int W, int PATHS>
__device__ __noinline__ bool batch_tile(const SampleJob &j, int64_t s0, uint64_t *bar, uint8_t *slots, uint32_t &g,
                                        uint8_t *scratch)
{
    return sample_tile<W, true, false, batch_spt(W, PATHS), PATHS>(j, s0, bar, slots, g, scratch);
}

// Class 0 (W <= 4): 128 registers, two CTAs of 256 threads per SM: on the
// mixed benchmark batch (32-bit, hybrid and general bodies in one launch) the
// fastest of the measured shapes (96 registers with five CTAs of 128, or with
// one shot per thread for the hybrid bodies, ran 10-20 % slower); class 1
// (W 5..16): the general body at up to 255.
#ifndef KSIM_BATCH_MAXNREG
#define KSIM_BATCH_MAXNREG 128
#endif
#define KSIM_BATCH_BOUNDS(C) __maxnreg__((C) == 0 ? KSIM_BATCH_MAXNREG : 255)
template <int CLASS>
__global__ void KSIM_BATCH_BOUNDS(CLASS) k_batch(const BatchJobDev *__restrict__ jobs,
                                                 const BatchItem *__restrict__ items, int n_items, int *counter)
{
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ int s_item;
    uint64_t *bar = (uint64_t *)smem;
    uint8_t *slots = smem + BAR_BYTES;
    ring_init(bar);
    uint32_t g = 0;
    uint8_t *scratch = slots + (size_t)NSLOT * jobs[0].j.slot_bytes;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int it = s_item;
        __syncthreads();
        if (it >= n_items) break;
        const BatchItem w = items[it];
        const BatchJobDev &J = jobs[w.job];
        bool ok = true;
        if (CLASS == 0) {
            // each job takes the body compiled for the term paths it uses
#define KSIM_BATCH_W(WW)                                                                              \
    case WW:                                                                                          \
        ok = J.paths == PATHS_NARROW ? batch_tile<WW, PATHS_NARROW>(J.j, w.s0, bar, slots, g, scratch) \
             : J.paths == PATHS_NARROW_HYBRID                                                         \
                 ? batch_tile<WW, PATHS_NARROW_HYBRID>(J.j, w.s0, bar, slots, g, scratch)            \
                 : batch_tile<WW, PATHS_ALL>(J.j, w.s0, bar, slots, g, scratch);                     \
        break;
            switch (J.W) {
            KSIM_BATCH_W(1) KSIM_BATCH_W(2) KSIM_BATCH_W(3)
            default: KSIM_BATCH_W(4)
            }
#undef KSIM_BATCH_W
        } else {
            switch (J.W) {
            case 5: ok = sample_tile<5, true, false, shots_per_thread(5)>(J.j, w.s0, bar, slots, g, scratch); break;
            case 6: ok = sample_tile<6, true, false, shots_per_thread(6)>(J.j, w.s0, bar, slots, g, scratch); break;
            case 8: ok = sample_tile<8, true, false, shots_per_thread(8)>(J.j, w.s0, bar, slots, g, scratch); break;
            case 10: ok = sample_tile<10, true, false, shots_per_thread(10)>(J.j, w.s0, bar, slots, g, scratch); break;
            case 12: ok = sample_tile<12, true, false, shots_per_thread(12)>(J.j, w.s0, bar, slots, g, scratch); break;
            default: ok = sample_tile<16, true, false, shots_per_thread(16)>(J.j, w.s0, bar, slots, g, scratch); break;
            }
        }
        if (!ok) break;
    }
}

}  // namespace

}  // namespace ksim

using namespace ksim;

struct ksim_batch {
    int device = 0;
    int threads = 256, slot_bytes = 16384, ctas_per_sm = 0, use_graph = 1;
    int max_w[2] = {1, 5};  // largest W among each class's jobs (parity scratch size)
    std::vector<ksim_component *> comps;
    std::vector<BatchJobDev> host_jobs;
    BatchJobDev *d_jobs = nullptr;
    BatchItem *d_items[2] = {nullptr, nullptr};
    int n_items[2] = {0, 0};
    int grid[2] = {0, 0};
    int *d_counter = nullptr;
    cudaStream_t cap_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

static ksim_status batch_enqueue(ksim_batch *b, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(b->d_counter, 0, 2 * sizeof(int), st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(work counter)");
    for (int cls = 0; cls < 2; ++cls) {
        if (!b->n_items[cls]) continue;
        const size_t smem = batch_smem_bytes(b->slot_bytes, b->max_w[cls], b->threads);
        if (cls == 0)
            k_batch<0><<<b->grid[0], b->threads, smem, st>>>(b->d_jobs, b->d_items[0], b->n_items[0], b->d_counter);
        else
            k_batch<1><<<b->grid[1], b->threads, smem, st>>>(b->d_jobs, b->d_items[1], b->n_items[1],
                                                             b->d_counter + 1);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "batch kernel launch");
    }
    return KSIM_OK;
}

extern "C" {

ksim_status ksim_batch_create(const ksim_batch_job *jobs, int32_t n_jobs, const ksim_batch_tuning *tuning,
                              ksim_batch **out)
{
    if (!out) return fail(KSIM_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (n_jobs <= 0 || !jobs) return fail(KSIM_ERR_INVALID_ARGUMENT, "a batch needs at least one job");
    std::unique_ptr<ksim_batch> b(new ksim_batch());
    if (tuning) {
        if (tuning->threads > 0) b->threads = tuning->threads;
        if (tuning->slot_bytes > 0) b->slot_bytes = tuning->slot_bytes;
        b->ctas_per_sm = tuning->ctas_per_sm;
        b->use_graph = tuning->use_graph;
    }
    if (b->threads > 256 || (b->threads & 31))
        return fail(KSIM_ERR_INVALID_ARGUMENT, "threads must be a multiple of 32 in [32, 256]");
    if ((b->slot_bytes & 15) || batch_smem_bytes(b->slot_bytes, 4, b->threads) > 227 * 1024)
        return fail(KSIM_ERR_INVALID_ARGUMENT,
                    "slot_bytes must be a multiple of 16, and two slots with the parity scratch fit in 227 KiB");
    int device = -1;
    for (int i = 0; i < n_jobs; ++i) {
        const ksim_batch_job &jb = jobs[i];
        ksim_component *c = jb.comp;
        if (!c) return fail(KSIM_ERR_INVALID_ARGUMENT, "job " + std::to_string(i) + ": component is NULL");
        if (device >= 0 && c->device != device)
            return fail(KSIM_ERR_INVALID_ARGUMENT, "jobs use components on different devices");
        device = c->device;
        if (jb.B < 0 || jb.shot_offset < 0)
            return fail(KSIM_ERR_INVALID_ARGUMENT, "job " + std::to_string(i) + ": negative B or offset");
        if (jb.rng_mode != KSIM_RNG_XORSHIFT && jb.rng_mode != KSIM_RNG_PHILOX)
            return fail(KSIM_ERR_INVALID_ARGUMENT, "job " + std::to_string(i) + ": bad rng_mode");
        if (jb.B > 0 && ((c->img.F > 0 && !jb.d_f) || (c->img.n_out > 0 && !jb.d_out)))
            return fail(KSIM_ERR_INVALID_ARGUMENT, "job " + std::to_string(i) + ": NULL buffer");
        if (c->img.max_term_bytes > b->slot_bytes)
            return fail(KSIM_ERR_INVALID_ARGUMENT, "job " + std::to_string(i) + ": a term record (" +
                                                       std::to_string(c->img.max_term_bytes) +
                                                       " bytes) exceeds slot_bytes");
        if (!jb.d_out_cols && jb.out_stride < jb.out_col0 + c->img.n_out)
            return fail(KSIM_ERR_INVALID_ARGUMENT, "job " + std::to_string(i) + ": out_stride too small");
    }
    b->device = device;
    DeviceGuard g(device);
    LaunchCfg cfg;
    cfg.threads = b->threads;
    cfg.staged = 1;
    cfg.slot_bytes = b->slot_bytes;
    std::vector<BatchItem> items[2];
    std::vector<double> cost[2];
    for (int i = 0; i < n_jobs; ++i) {
        const ksim_batch_job &jb = jobs[i];
        ksim_component *c = jb.comp;
        BatchJobDev d = {};
        ksim_status st = component_job(c, cfg, d.j);
        if (st != KSIM_OK) return st;
        d.j.rng_mode = jb.rng_mode;
        d.j.f = jb.d_f;
        d.j.f_stride = jb.f_stride;
        d.j.f_sel = jb.d_f_sel;
        d.j.out = jb.d_out;
        d.j.out_stride = jb.out_stride;
        d.j.out_col0 = jb.out_col0;
        d.j.out_cols = jb.d_out_cols;
        d.j.amp = nullptr;
        d.j.B = jb.B;
        d.j.shot_offset = jb.shot_offset;
        d.j.seed = jb.seed;
        d.W = c->img.W;
        d.paths = c->cfg.paths;
        b->host_jobs.push_back(d);
        b->comps.push_back(c);
        if (c->img.n_out == 0 || jb.B == 0) continue;
        double bytes = 0;
        for (const GraphDir &gd : c->img.gdir) bytes += (double)gd.stream_bytes + 64.0;
        const int cls = d.W <= 4 ? 0 : 1;
        b->max_w[cls] = std::max(b->max_w[cls], d.W);
        const int64_t tile = (int64_t)b->threads * batch_spt(d.W, d.paths);
        for (int64_t s0 = 0; s0 < jb.B; s0 += tile) {
            BatchItem it = {};
            it.job = i;
            it.s0 = s0;
            items[cls].push_back(it);
            cost[cls].push_back(bytes * (double)std::min<int64_t>(tile, jb.B - s0));
        }
    }
    cudaError_t e = cudaMalloc(&b->d_jobs, sizeof(BatchJobDev) * b->host_jobs.size());
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_jobs, b->host_jobs.data(), sizeof(BatchJobDev) * b->host_jobs.size(),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_counter, 2 * sizeof(int));
    if (e != cudaSuccess) {
        ksim_batch_destroy(b.release());
        return cuda_fail(e, "batch upload");
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    for (int cls = 0; cls < 2; ++cls) {
        const size_t smem = batch_smem_bytes(b->slot_bytes, b->max_w[cls], b->threads);
        std::vector<int> order(items[cls].size());
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost[cls][x] > cost[cls][y]; });
        std::vector<BatchItem> sorted;
        sorted.reserve(order.size());
        for (int o : order) sorted.push_back(items[cls][o]);
        b->n_items[cls] = (int)sorted.size();
        if (sorted.empty()) continue;
        e = cudaMalloc(&b->d_items[cls], sizeof(BatchItem) * sorted.size());
        if (e == cudaSuccess)
            e = cudaMemcpy(b->d_items[cls], sorted.data(), sizeof(BatchItem) * sorted.size(), cudaMemcpyHostToDevice);
        int active = 0;
        if (e == cudaSuccess) {
            const void *fn = cls == 0 ? (const void *)k_batch<0> : (const void *)k_batch<1>;
            e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&active, fn, b->threads, smem);
        }
        if (e != cudaSuccess) {
            ksim_batch_destroy(b.release());
            return cuda_fail(e, "batch setup");
        }
        const int per_sm = b->ctas_per_sm > 0 ? std::min(b->ctas_per_sm, std::max(active, 1)) : std::max(active, 1);
        b->grid[cls] = std::max(1, std::min(per_sm * sms, b->n_items[cls]));
    }
    *out = b.release();
    return KSIM_OK;
}

ksim_status ksim_batch_set_seeds(ksim_batch *b, const uint64_t *seeds)
{
    if (!b || !seeds) return fail(KSIM_ERR_INVALID_ARGUMENT, "batch or seeds is NULL");
    DeviceGuard g(b->device);
    for (size_t i = 0; i < b->host_jobs.size(); ++i) b->host_jobs[i].j.seed = seeds[i];
    cudaError_t e = cudaMemcpy(b->d_jobs, b->host_jobs.data(), sizeof(BatchJobDev) * b->host_jobs.size(),
                               cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "batch seeds");
    return KSIM_OK;
}

ksim_status ksim_batch_launch(ksim_batch *b, void *stream)
{
    if (!b) return fail(KSIM_ERR_INVALID_ARGUMENT, "batch is NULL");
    DeviceGuard g(b->device);
    cudaStream_t st = (cudaStream_t)stream;
    if (!b->use_graph) return batch_enqueue(b, st);
    if (!b->exec) {
        cudaError_t e = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
        e = cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamBeginCapture");
        ksim_status s = batch_enqueue(b, b->cap_stream);
        e = cudaStreamEndCapture(b->cap_stream, &b->graph);
        if (s != KSIM_OK) return s;
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&b->exec, b->graph, 0);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
    }
    cudaError_t e = cudaGraphLaunch(b->exec, st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
    return KSIM_OK;
}

ksim_status ksim_batch_info(const ksim_batch *b, int64_t *n_items, int32_t *grid, int32_t *n_launches)
{
    if (!b) return fail(KSIM_ERR_INVALID_ARGUMENT, "batch is NULL");
    if (n_items) *n_items = (int64_t)b->n_items[0] + b->n_items[1];
    if (grid) *grid = b->grid[0] + b->grid[1];
    if (n_launches) *n_launches = (b->n_items[0] ? 1 : 0) + (b->n_items[1] ? 1 : 0);
    return KSIM_OK;
}

void ksim_batch_destroy(ksim_batch *b)
{
    if (!b) return;
    DeviceGuard g(b->device);
    cudaDeviceSynchronize();
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
    for (int c = 0; c < 2; ++c)
        if (b->d_items[c]) cudaFree(b->d_items[c]);
    if (b->d_jobs) cudaFree(b->d_jobs);
    if (b->d_counter) cudaFree(b->d_counter);
    delete b;
}

}  // extern "C"
