// batch.cu — many components / programs in one graph-captured launch of
// persistent kernels.
//
// Work is cut into items (job, tile of shots).  Items are ordered
// longest-first (cost = tile shots x term-stream bytes of the job's component)
// and persistent CTAs pull them from a device work counter with one
// atomicAdd per item, so programs with uneven term counts, output counts and
// shot counts share the GPU with little tail.  A CTA keeps one staging ring
// for its whole life; its running chunk count picks each copy's slot and
// barrier phase across items of different jobs.
//
// Items are grouped into classes by the kernel body their job needs: (W, term
// paths) for W <= 4 — 32-bit, hybrid or general (64-bit words / exact path)
// bodies — and one class for W in 5..16.  Each class present in a batch is
// drained by its own persistent kernel compiled with that one body inline
// and no out-of-line calls (a kernel that holds several bodies, or calls
// between them, ran 6-11 % slower on the same items), with the register
// budget of the plain kernel for that body.  The job table travels in the
// kernels' parameter space when it fits (BATCH_PARAM_JOBS jobs), so job fields
// are read from the constant bank as in the plain kernel, otherwise from
// global memory.  The class kernels go on one stream in a fixed order — the
// hybrid, general and wide classes (the heaviest items) first, then the
// 32-bit ones, each group by its costliest item — as programmatic dependent
// launches: each kernel starts once every CTA of the one before it runs, and
// fills the slots that one frees as it drains, so the classes overlap without
// the run-to-run dispatch order of concurrent graph branches.  The counter
// reset and the launches are captured once into a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
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

// Classes: 3 (W - 1) + p for W <= 4 (p = 0 32-bit, 1 hybrid, 2 general), 12
// for W > 4.
constexpr int BATCH_CLASSES = 13;
constexpr int BATCH_WIDE = 12;
inline int batch_class(int W, int paths)
{
    if (W > 4) return BATCH_WIDE;
    const int p = paths == PATHS_NARROW ? 0 : paths == PATHS_NARROW_HYBRID ? 1 : 2;
    return 3 * (W - 1) + p;
}

namespace {

// The parity scratch is sized for the largest W among a class's jobs
// (smaller scratch leaves more of the SM's shared storage to L1).
size_t batch_smem_bytes(int slot_bytes, int max_w, int threads)
{
    return sample_smem_bytes(slot_bytes, true, max_w, threads);
}

// One launch's view of the batch: its class's items and counter, its staging
// slot, and the job table by value (BatchParams, up to BATCH_PARAM_JOBS jobs)
// or through a pointer (BatchParamsG).
constexpr int BATCH_PARAM_JOBS = 180;
struct BatchParams {
    const BatchItem *items;
    int *counter;
    int32_t n_items, slot_bytes;
    BatchJobDev jobs[BATCH_PARAM_JOBS];
    __device__ __forceinline__ const BatchJobDev &job(int i) const { return jobs[i]; }
};
static_assert(sizeof(BatchParams) <= 32764, "kernel parameters are limited to 32,764 bytes");
struct BatchParamsG {
    const BatchItem *items;
    int *counter;
    int32_t n_items, slot_bytes;
    const BatchJobDev *gjobs;
    __device__ __forceinline__ const BatchJobDev &job(int i) const { return gjobs[i]; }
};

// CTA sizes of the hybrid and of the general / wide classes.  Their items
// are the heaviest (up to a few times a 32-bit item's work per shot), and a
// smaller CTA is a shorter item, so the last ones end sooner; these jobs also
// tend to have few shots, and 128-thread CTAs spread them over four times the
// SMs of 256-thread ones (a 57-qubit, 11,170-shot general job: 1.78 against
// 2.22 ms alone on the GPU).
#ifndef KSIM_BATCH_HYB_THREADS
#define KSIM_BATCH_HYB_THREADS 128
#endif
#ifndef KSIM_BATCH_GEN_THREADS
#define KSIM_BATCH_GEN_THREADS 128
#endif

// Register budgets: those of the plain kernels for the 32-bit and hybrid
// bodies (96), four CTAs of 128 for the general body (128).
#define KSIM_BATCH_BOUNDS(P) __maxnreg__((P) == PATHS_ALL ? 128 : 96)

// Programmatic dependent launch: the class kernels are launched on one
// stream, heaviest class first, each allowed to start once every CTA of the
// previous one runs (launch_dependents, at a CTA's start), so they overlap and
// a later class fills the slots the earlier ones leave; before leaving, a CTA
// waits until the previous class's kernel has finished (wait), so the stream
// still completes in launch order.  A kernel starts only after all CTAs of
// its predecessor are resident, so the wait never holds slots its
// predecessor needs.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// A class with W <= 4: one body, inline.
template <typename PT, int W, int PATHS>
__global__ void KSIM_BATCH_BOUNDS(PATHS) k_batch_c(const __grid_constant__ PT P)
{
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ int s_item;
    uint64_t *bar = (uint64_t *)smem;
    uint8_t *slots = smem + BAR_BYTES;
    ring_init(bar);
    pdl_launch_dependents();
    uint32_t g = 0;
    uint8_t *scratch = slots + (size_t)NSLOT * P.slot_bytes;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(P.counter, 1);
        __syncthreads();
        const int it = s_item;
        __syncthreads();
        if (it >= P.n_items) break;
        const BatchItem w = P.items[it];
        if (!sample_tile<W, true, false, shots_per_thread(W), PATHS>(P.job(w.job).j, w.s0, bar, slots, g, scratch))
            break;
    }
    pdl_wait();
}

// The class with W in 5..16 (rare): the general body per W.
template <typename PT>
__global__ void __maxnreg__(255) k_batch_wide(const __grid_constant__ PT P)
{
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ int s_item;
    uint64_t *bar = (uint64_t *)smem;
    uint8_t *slots = smem + BAR_BYTES;
    ring_init(bar);
    pdl_launch_dependents();
    uint32_t g = 0;
    uint8_t *scratch = slots + (size_t)NSLOT * P.slot_bytes;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(P.counter, 1);
        __syncthreads();
        const int it = s_item;
        __syncthreads();
        if (it >= P.n_items) break;
        const BatchItem w = P.items[it];
        const BatchJobDev &J = P.job(w.job);
        bool ok;
        switch (J.W) {
        case 5: ok = sample_tile<5, true, false, shots_per_thread(5)>(J.j, w.s0, bar, slots, g, scratch); break;
        case 6: ok = sample_tile<6, true, false, shots_per_thread(6)>(J.j, w.s0, bar, slots, g, scratch); break;
        case 8: ok = sample_tile<8, true, false, shots_per_thread(8)>(J.j, w.s0, bar, slots, g, scratch); break;
        case 10: ok = sample_tile<10, true, false, shots_per_thread(10)>(J.j, w.s0, bar, slots, g, scratch); break;
        case 12: ok = sample_tile<12, true, false, shots_per_thread(12)>(J.j, w.s0, bar, slots, g, scratch); break;
        default: ok = sample_tile<16, true, false, shots_per_thread(16)>(J.j, w.s0, bar, slots, g, scratch); break;
        }
        if (!ok) break;
    }
    pdl_wait();
}

// The kernel of class `cls` for job-table type PT.
template <typename PT>
const void *batch_kernel(int cls)
{
#define KSIM_BK(WW)                                                                  \
    case 3 * (WW - 1): return (const void *)k_batch_c<PT, WW, PATHS_NARROW>;         \
    case 3 * (WW - 1) + 1: return (const void *)k_batch_c<PT, WW, PATHS_NARROW_HYBRID>; \
    case 3 * (WW - 1) + 2: return (const void *)k_batch_c<PT, WW, PATHS_ALL>;
    switch (cls) {
    KSIM_BK(1) KSIM_BK(2) KSIM_BK(3) KSIM_BK(4)
    default: return (const void *)k_batch_wide<PT>;
    }
#undef KSIM_BK
}

}  // namespace

}  // namespace ksim

using namespace ksim;

namespace {

// One class of a batch: launch shape and items.
struct BatchClass {
    int threads = 128, slot = 14336, max_w = 1;
    size_t smem = 0;
    BatchItem *d_items = nullptr;
    int n_items = 0, grid = 0;
    bool high = false;      // hybrid, general and wide classes: launched before the 32-bit ones
    double head_cost = 0;   // cost of its costliest item
    std::unique_ptr<BatchParams> p;  // the job table by value (<= BATCH_PARAM_JOBS jobs)
    BatchParamsG pg = {};            // otherwise through a pointer
};

}  // namespace

struct ksim_batch {
    int device = 0;
    int threads = 128, slot_bytes = 14336, ctas_per_sm = 0, use_graph = 1;  // 32-bit classes (tuned)
    BatchClass cls[BATCH_CLASSES];
    std::vector<ksim_component *> comps;
    std::vector<BatchJobDev> host_jobs;
    BatchJobDev *d_jobs = nullptr;
    int *d_counter = nullptr;
    cudaStream_t cap_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

// Drop the captured graph (its kernel nodes hold the job table by value).
static void batch_drop_graph(ksim_batch *b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

// Launch class c's kernel on `st`; `follow`: it may start as soon as every CTA
// of the kernel launched before it on `st` runs (programmatic dependent launch).
static cudaError_t batch_launch_class(ksim_batch *b, int c, cudaStream_t st, bool follow)
{
    BatchClass &k = b->cls[c];
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3((unsigned)k.grid);
    lc.blockDim = dim3((unsigned)k.threads);
    lc.dynamicSmemBytes = k.smem;
    lc.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    lc.attrs = at;
    lc.numAttrs = follow ? 1 : 0;
    if (k.p) {
        void *args[] = {(void *)k.p.get()};
        return cudaLaunchKernelExC(&lc, batch_kernel<BatchParams>(c), args);
    }
    void *args[] = {(void *)&k.pg};
    return cudaLaunchKernelExC(&lc, batch_kernel<BatchParamsG>(c), args);
}

static ksim_status batch_enqueue(ksim_batch *b, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(b->d_counter, 0, BATCH_CLASSES * sizeof(int), st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(work counter)");
    // the hybrid / general / wide classes first, then the 32-bit ones; within
    // each group the class with the costliest first item first
    std::vector<int> active;
    for (int c = 0; c < BATCH_CLASSES; ++c)
        if (b->cls[c].n_items) active.push_back(c);
    std::stable_sort(active.begin(), active.end(), [&](int x, int y) {
        const BatchClass &a = b->cls[x], &z = b->cls[y];
        if (a.high != z.high) return a.high;
        return a.head_cost > z.head_cost;
    });
    for (size_t i = 0; i < active.size(); ++i)
        if ((e = batch_launch_class(b, active[i], st, i > 0)) != cudaSuccess)
            return cuda_fail(e, "batch kernel launch");
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
    const bool slot_given = tuning && tuning->slot_bytes > 0;
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
    // shapes: the 32-bit classes the tuned one; hybrid CTAs of
    // KSIM_BATCH_HYB_THREADS, general and wide CTAs of KSIM_BATCH_GEN_THREADS;
    // slots at least the tuned size (16 KiB for general and wide) and every
    // job's largest term
    for (int c = 0; c < BATCH_CLASSES; ++c) {
        BatchClass &k = b->cls[c];
        const int p = c == BATCH_WIDE ? 3 : c % 3;
        k.threads = p == 0 ? b->threads : p == 1 ? KSIM_BATCH_HYB_THREADS : KSIM_BATCH_GEN_THREADS;
        k.slot = p >= 2 ? std::max(16384, b->slot_bytes) : b->slot_bytes;
        k.high = p != 0;
        k.max_w = c == BATCH_WIDE ? 5 : c / 3 + 1;
    }
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
        if (!jb.d_out_cols && jb.out_stride < jb.out_col0 + c->img.n_out)
            return fail(KSIM_ERR_INVALID_ARGUMENT, "job " + std::to_string(i) + ": out_stride too small");
        const int cl = batch_class(c->img.W, c->cfg.paths);
        BatchClass &k = b->cls[cl];
        const int64_t need = (c->img.max_term_bytes + 15) & ~int64_t(15);
        // a slot the caller chose must hold the 32-bit jobs' terms; the
        // default and the other classes' slots grow to their largest term
        if (slot_given && cl % 3 == 0 && cl != BATCH_WIDE && need > b->slot_bytes)
            return fail(KSIM_ERR_INVALID_ARGUMENT, "job " + std::to_string(i) + ": a term record (" +
                                                       std::to_string(c->img.max_term_bytes) +
                                                       " bytes) exceeds slot_bytes");
        if (need > k.slot) k.slot = (int)std::min<int64_t>(need, 1 << 30);
        k.max_w = std::max(k.max_w, c->img.W);
    }
    for (int c = 0; c < BATCH_CLASSES; ++c)
        if (batch_smem_bytes(b->cls[c].slot, b->cls[c].max_w, b->cls[c].threads) > 227 * 1024)
            return fail(KSIM_ERR_UNSUPPORTED, "a term record needs a staging slot of " +
                                                  std::to_string(b->cls[c].slot) + " bytes, beyond shared memory");
    b->device = device;
    DeviceGuard g(device);
    std::vector<BatchItem> items[BATCH_CLASSES];
    std::vector<double> cost[BATCH_CLASSES];
    for (int i = 0; i < n_jobs; ++i) {
        const ksim_batch_job &jb = jobs[i];
        ksim_component *c = jb.comp;
        const int cl = batch_class(c->img.W, c->cfg.paths);
        BatchClass &k = b->cls[cl];
        LaunchCfg cfg;
        cfg.threads = k.threads;
        cfg.staged = 1;
        cfg.slot_bytes = k.slot;
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
        const int64_t tile = (int64_t)k.threads * shots_per_thread(d.W);
        for (int64_t s0 = 0; s0 < jb.B; s0 += tile) {
            BatchItem it = {};
            it.job = i;
            it.s0 = s0;
            items[cl].push_back(it);
            cost[cl].push_back(bytes * (double)std::min<int64_t>(tile, jb.B - s0));
        }
    }
    cudaError_t e = cudaMalloc(&b->d_jobs, sizeof(BatchJobDev) * b->host_jobs.size());
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_jobs, b->host_jobs.data(), sizeof(BatchJobDev) * b->host_jobs.size(),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_counter, BATCH_CLASSES * sizeof(int));
    if (e != cudaSuccess) {
        ksim_batch_destroy(b.release());
        return cuda_fail(e, "batch upload");
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const bool by_value = b->host_jobs.size() <= (size_t)BATCH_PARAM_JOBS;
    for (int c = 0; c < BATCH_CLASSES; ++c) {
        BatchClass &k = b->cls[c];
        if (items[c].empty()) continue;
        k.smem = batch_smem_bytes(k.slot, k.max_w, k.threads);
        std::vector<int> order(items[c].size());
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost[c][x] > cost[c][y]; });
        std::vector<BatchItem> sorted;
        sorted.reserve(order.size());
        for (int o : order) sorted.push_back(items[c][o]);
        k.n_items = (int)sorted.size();
        k.head_cost = cost[c][order[0]];
        e = cudaMalloc(&k.d_items, sizeof(BatchItem) * sorted.size());
        if (e == cudaSuccess)
            e = cudaMemcpy(k.d_items, sorted.data(), sizeof(BatchItem) * sorted.size(), cudaMemcpyHostToDevice);
        if (by_value) {
            k.p.reset(new BatchParams());
            std::memset(k.p.get(), 0, sizeof(BatchParams));
            k.p->items = k.d_items;
            k.p->counter = b->d_counter + c;
            k.p->n_items = k.n_items;
            k.p->slot_bytes = k.slot;
            std::copy(b->host_jobs.begin(), b->host_jobs.end(), k.p->jobs);
        } else {
            k.pg.items = k.d_items;
            k.pg.counter = b->d_counter + c;
            k.pg.n_items = k.n_items;
            k.pg.slot_bytes = k.slot;
            k.pg.gjobs = b->d_jobs;
        }
        int active = 0;
        if (e == cudaSuccess) {
            const void *fn = by_value ? batch_kernel<BatchParams>(c) : batch_kernel<BatchParamsG>(c);
            e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem);
            if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&active, fn, k.threads, k.smem);
        }
        if (e != cudaSuccess) {
            ksim_batch_destroy(b.release());
            return cuda_fail(e, "batch setup");
        }
        const int per_sm = (c % 3 == 0 && c != BATCH_WIDE && b->ctas_per_sm > 0)
                               ? std::min(b->ctas_per_sm, std::max(active, 1))
                               : std::max(active, 1);
        k.grid = std::max(1, std::min(per_sm * sms, k.n_items));
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
    bool by_value = false;
    for (BatchClass &k : b->cls)
        if (k.p) {
            by_value = true;
            for (size_t i = 0; i < b->host_jobs.size(); ++i) k.p->jobs[i].j.seed = seeds[i];
        }
    if (by_value) batch_drop_graph(b);  // recaptured with the new seeds on the next launch
    return KSIM_OK;
}

ksim_status ksim_batch_launch(ksim_batch *b, void *stream)
{
    if (!b) return fail(KSIM_ERR_INVALID_ARGUMENT, "batch is NULL");
    DeviceGuard g(b->device);
    cudaStream_t st = (cudaStream_t)stream;
    if (!b->use_graph) return batch_enqueue(b, st);
    if (!b->exec) {
        cudaError_t e = cudaSuccess;
        if (!b->cap_stream) e = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
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
    int64_t n = 0;
    int32_t gsum = 0, l = 0;
    for (const BatchClass &k : b->cls)
        if (k.n_items) {
            n += k.n_items;
            gsum += k.grid;
            ++l;
        }
    if (n_items) *n_items = n;
    if (grid) *grid = gsum;
    if (n_launches) *n_launches = l;
    return KSIM_OK;
}

void ksim_batch_destroy(ksim_batch *b)
{
    if (!b) return;
    DeviceGuard g(b->device);
    cudaDeviceSynchronize();
    batch_drop_graph(b);
    if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
    for (BatchClass &k : b->cls) {
        if (k.d_items) cudaFree(k.d_items);
    }
    if (b->d_jobs) cudaFree(b->d_jobs);
    if (b->d_counter) cudaFree(b->d_counter);
    delete b;
}

}  // extern "C"
