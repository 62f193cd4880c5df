// api.cu — the C ABI (include/ksim_b200.h): components, programs, launches.
//
// A component owns its device program image (uploaded once, like the
// reference's four Kokkos Views, kokkos_sim.cpp:132-149), one chunk directory
// per staging slot size, a status word, a stream for the synchronous host
// calls and grow-only device workspaces for those calls.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/ksim_b200.h"
#include "hostio.h"
#include "image.h"
#include "kernels.h"
#include "runtime.h"

namespace ksim {

thread_local std::string g_err;

ksim_status fail(ksim_status s, const std::string &m)
{
    g_err = m;
    return s;
}

ksim_status cuda_fail(cudaError_t e, const char *what)
{
    return fail(e == cudaErrorMemoryAllocation ? KSIM_ERR_OUT_OF_MEMORY : KSIM_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

DeviceGuard::DeviceGuard(int dev)
{
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (dev >= 0 && dev != prev) ok = cudaSetDevice(dev) == cudaSuccess;
}
DeviceGuard::~DeviceGuard()
{
    if (prev >= 0) cudaSetDevice(prev);
}

cudaError_t DevBuf::ensure(size_t n)
{
    if (n <= cap) return cudaSuccess;
    release();
    cudaError_t e = cudaMalloc(&p, n);
    if (e == cudaSuccess) cap = n;
    else p = nullptr;
    return e;
}
void DevBuf::release()
{
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
}

ksim_status component_chunks(ksim_component *c, int slot_bytes, const ChunkDir **d, int *n)
{
    std::lock_guard<std::mutex> lk(c->chunk_mu);
    auto it = c->chunks.find(slot_bytes);
    if (it == c->chunks.end()) {
        std::vector<ChunkDir> host;
        if (!make_chunks(c->img, slot_bytes, host))
            return fail(KSIM_ERR_INVALID_ARGUMENT, "slot_bytes " + std::to_string(slot_bytes) +
                                                       " is smaller than the largest term record (" +
                                                       std::to_string(c->img.max_term_bytes) + ")");
        ComponentChunks cc;
        cc.n = (int)host.size();
        cudaError_t e = cudaMalloc(&cc.d, host.size() * sizeof(ChunkDir));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(chunk directory)");
        e = cudaMemcpy(cc.d, host.data(), host.size() * sizeof(ChunkDir), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(cc.d);
            return cuda_fail(e, "cudaMemcpy(chunk directory)");
        }
        it = c->chunks.emplace(slot_bytes, cc).first;
    }
    *d = it->second.d;
    *n = it->second.n;
    return KSIM_OK;
}

// After a synchronous call: KSIM_ERR_TIMEOUT if a staging wait of the
// component's kernels ran out, clearing that flag (the other flags stay for
// ksim_component_status).
// A component's status word as read after a call (`flags`): a wait that
// ran out fails the call and is cleared from the word (the other flags stay
// for ksim_component_status).
ksim_status report_timeout_flags(ksim_component *c, uint32_t flags)
{
    if (!(flags & KSIM_FLAG_WAIT_TIMEOUT)) return KSIM_OK;
    const uint32_t rest = flags & ~(uint32_t)KSIM_FLAG_WAIT_TIMEOUT;
    const cudaError_t e = cudaMemcpy(c->d_status, &rest, sizeof(rest), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "status write");
    return fail(KSIM_ERR_TIMEOUT, "a staging wait of the sampling kernel ran out; its shots were not written");
}

ksim_status report_timeout(ksim_component *c)
{
    uint32_t flags = 0;
    cudaError_t e = cudaMemcpy(&flags, c->d_status, sizeof(flags), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "status read");
    return report_timeout_flags(c, flags);
}

// Fill a SampleJob for component c; inputs/outputs set by the caller.
ksim_status component_job(ksim_component *c, const LaunchCfg &cfg, SampleJob &j)
{
    const ChunkDir *cd = nullptr;
    int nc = 0;
    const int slot = cfg.staged ? cfg.slot_bytes : (int)std::max<int64_t>(c->img.max_term_bytes, 16);
    ksim_status st = component_chunks(c, cfg.staged ? cfg.slot_bytes : (1 << 30), &cd, &nc);
    if (st != KSIM_OK) return st;
    j.image = c->d_image;
    j.gdir = (const GraphDir *)c->d_image;
    j.cdir = cd;
    j.n_chunks = nc;
    j.n_graphs = c->img.n_graphs;
    j.F = c->img.F;
    j.n_out = c->img.n_out;
    j.slot_bytes = slot;
    j.status = c->d_status;
    j.wait_limit = c->wait_limit;
    return KSIM_OK;
}

}  // namespace ksim

namespace {
// Host buffers in and out of a program, chunked and copy-overlapped (below).
ksim_status program_sample_host(ksim_program *p, const uint8_t *f, int64_t B, int64_t n_f_cols, uint64_t seed,
                                int32_t rng_mode, uint8_t *out, bool packed, const ksim_noise *noise = nullptr,
                                uint64_t noise_seed = 0);
}  // namespace

using namespace ksim;

extern "C" {

const char *ksim_last_error(void) { return g_err.c_str(); }
int32_t ksim_abi_version(void) { return KSIM_B200_ABI_VERSION; }

int32_t ksim_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

ksim_status ksim_work_model(const ksim_graph_desc *graphs, int32_t n_graphs, int32_t num_f, double *ops_per_shot,
                            int64_t *paths)
{
    if (!ops_per_shot) return fail(KSIM_ERR_INVALID_ARGUMENT, "ops_per_shot is NULL");
    HostImage img;
    std::string err;
    int st = build_image(graphs, n_graphs, num_f, img, err);
    if (st != KSIM_OK) return fail((ksim_status)st, err);
    *ops_per_shot = img.work_ops;
    if (paths) {
        paths[0] = img.n_narrow_terms;
        paths[1] = img.n_terms - img.n_narrow_terms - img.n_slow_terms - img.n_hybrid_terms;
        paths[2] = img.n_slow_terms;
        paths[3] = img.n_hybrid_terms;
    }
    return KSIM_OK;
}

ksim_status ksim_component_create(const ksim_graph_desc *graphs, int32_t n_graphs, int32_t num_f,
                                  int32_t device, ksim_component **out)
{
    if (!out) return fail(KSIM_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (ksim_device_count() <= 0) return fail(KSIM_ERR_NO_DEVICE, "no CUDA device is visible");
    std::unique_ptr<ksim_component> c(new ksim_component());
    std::string err;
    int st = build_image(graphs, n_graphs, num_f, c->img, err);
    if (st != KSIM_OK) return fail((ksim_status)st, err);
    if (device < 0) {
        if (cudaGetDevice(&device) != cudaSuccess) return fail(KSIM_ERR_NO_DEVICE, "cudaGetDevice failed");
    }
    c->device = device;
    DeviceGuard g(device);
    if (!g.ok) return fail(KSIM_ERR_INVALID_ARGUMENT, "cannot select device " + std::to_string(device));
    cudaError_t e = cudaMalloc(&c->d_image, c->img.bytes.size());
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(program image)");
    c->image_bytes = c->img.bytes.size();
    e = cudaMemcpy(c->d_image, c->img.bytes.data(), c->img.bytes.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy(program image)");
    e = cudaMalloc(&c->d_status, sizeof(uint32_t));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(status)");
    e = cudaMemset(c->d_status, 0, sizeof(uint32_t));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemset(status)");
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
    // default launch shape: slot fits the largest term and at least 16 KiB;
    // staging is skipped when two slots would not fit in shared memory
    c->cfg.paths = c->img.n_narrow_terms == c->img.n_terms ? 1
                   : c->img.n_narrow_terms + c->img.n_hybrid_terms == c->img.n_terms ? 2 : 0;
    // slots for the specialised kernels as large as five CTAs per SM allow
    // (14 KiB for W <= 2, 12 KiB for W = 3, 4: fewer chunks per graph), 16 KiB
    // else
    const int64_t slot = std::max<int64_t>(c->cfg.paths != 0 ? (c->img.W <= 2 ? 14336 : 12288) : 16384,
                                           (c->img.max_term_bytes + 15) & ~int64_t(15));
    c->cfg.threads = 128;  // CTAs of 128: a quarter of the warps per barrier
    c->cfg.slot_bytes = (int)std::min<int64_t>(slot, 1 << 30);
    c->cfg.staged =
        sample_smem_bytes((int)std::min<int64_t>(slot, 1 << 20), true, c->img.W, c->cfg.threads) <= 200 * 1024 ? 1
                                                                                                            : 0;
    // free the packed bytes; term offsets stay for re-chunking
    c->img.bytes.clear();
    c->img.bytes.shrink_to_fit();
    *out = c.release();
    return KSIM_OK;
}

void ksim_component_destroy(ksim_component *c)
{
    if (!c) return;
    DeviceGuard g(c->device);
    if (c->self_prog) ksim_program_destroy(c->self_prog);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto &kv : c->chunks) cudaFree(kv.second.d);
    c->ws_f.release();
    c->ws_out.release();
    c->ws_aux.release();
    if (c->d_status) cudaFree(c->d_status);
    if (c->d_image) cudaFree(c->d_image);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

int32_t ksim_component_n_out(const ksim_component *c) { return c ? c->img.n_out : -1; }
int32_t ksim_component_num_f(const ksim_component *c) { return c ? c->img.F : -1; }
int32_t ksim_component_n_graphs(const ksim_component *c) { return c ? c->img.n_graphs : -1; }
int32_t ksim_component_words(const ksim_component *c) { return c ? c->img.W : -1; }
int64_t ksim_component_image_bytes(const ksim_component *c) { return c ? (int64_t)c->image_bytes : -1; }

ksim_status ksim_component_set_launch(ksim_component *c, int32_t threads, int32_t staged, int32_t slot_bytes)
{
    if (!c) return fail(KSIM_ERR_INVALID_ARGUMENT, "component is NULL");
    std::lock_guard<std::mutex> lk(c->mu);
    LaunchCfg cfg = c->cfg;
    if (threads > 0) {
        if (threads > 256 || (threads & 31))
            return fail(KSIM_ERR_INVALID_ARGUMENT, "threads must be a multiple of 32 in [32, 256]");
        cfg.threads = threads;
    }
    if (staged >= 0) cfg.staged = staged ? 1 : 0;
    if (slot_bytes > 0) {
        if ((slot_bytes & 15) || slot_bytes < c->img.max_term_bytes)
            return fail(KSIM_ERR_INVALID_ARGUMENT,
                        "slot_bytes must be a multiple of 16 and hold the largest term record (" +
                            std::to_string(c->img.max_term_bytes) + " bytes)");
        cfg.slot_bytes = slot_bytes;
    }
    if (sample_smem_bytes(cfg.slot_bytes, cfg.staged != 0, c->img.W, cfg.threads) > 227 * 1024)
        return fail(KSIM_ERR_INVALID_ARGUMENT,
                    "the staging slots and the parity scratch exceed 227 KiB of shared memory");
    c->cfg = cfg;
    return KSIM_OK;
}

ksim_status ksim_component_set_wait_limit(ksim_component *c, int64_t polls)
{
    if (!c) return fail(KSIM_ERR_INVALID_ARGUMENT, "component is NULL");
    if (polls < 0) return fail(KSIM_ERR_INVALID_ARGUMENT, "polls must be >= 0");
    std::lock_guard<std::mutex> lk(c->mu);
    c->wait_limit = polls;
    return KSIM_OK;
}

ksim_status ksim_component_get_launch(const ksim_component *c, int32_t *threads, int32_t *staged,
                                      int32_t *slot_bytes)
{
    if (!c) return fail(KSIM_ERR_INVALID_ARGUMENT, "component is NULL");
    if (threads) *threads = c->cfg.threads;
    if (staged) *staged = c->cfg.staged;
    if (slot_bytes) *slot_bytes = c->cfg.slot_bytes;
    return KSIM_OK;
}

ksim_status ksim_component_stats(const ksim_component *c, int64_t *n_terms, int64_t *n_slow_terms,
                                 int64_t *n_columns, int64_t *max_term_bytes)
{
    if (!c) return fail(KSIM_ERR_INVALID_ARGUMENT, "component is NULL");
    if (n_terms) *n_terms = c->img.n_terms;
    if (n_slow_terms) *n_slow_terms = c->img.n_slow_terms;
    if (n_columns) *n_columns = c->img.n_columns;
    if (max_term_bytes) *max_term_bytes = c->img.max_term_bytes;
    return KSIM_OK;
}

static ksim_status check_rng(int32_t rng_mode)
{
    if (rng_mode != KSIM_RNG_XORSHIFT && rng_mode != KSIM_RNG_PHILOX)
        return fail(KSIM_ERR_INVALID_ARGUMENT, "rng_mode must be KSIM_RNG_XORSHIFT or KSIM_RNG_PHILOX");
    return KSIM_OK;
}

ksim_status ksim_component_sample_device(ksim_component *c, const uint8_t *d_f_sel, int64_t B,
                                         int64_t shot_offset, uint64_t seed, int32_t rng_mode,
                                         uint8_t *d_out, int64_t out_stride, int64_t out_col0,
                                         double *d_amp, void *stream)
{
    if (!c) return fail(KSIM_ERR_INVALID_ARGUMENT, "component is NULL");
    if (B < 0 || shot_offset < 0) return fail(KSIM_ERR_INVALID_ARGUMENT, "B and shot_offset must be >= 0");
    if (check_rng(rng_mode) != KSIM_OK) return KSIM_ERR_INVALID_ARGUMENT;
    if (B == 0 || c->img.n_out == 0 && !d_amp) return KSIM_OK;
    if ((c->img.F > 0 && !d_f_sel) || (c->img.n_out > 0 && !d_out))
        return fail(KSIM_ERR_INVALID_ARGUMENT, "input or output pointer is NULL");
    if (out_col0 < 0 || out_stride < out_col0 + c->img.n_out)
        return fail(KSIM_ERR_INVALID_ARGUMENT, "out_stride must be >= out_col0 + n_out");
    DeviceGuard g(c->device);
    LaunchCfg cfg;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        cfg = c->cfg;
    }
    SampleJob j = {};
    ksim_status st = component_job(c, cfg, j);
    if (st != KSIM_OK) return st;
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
    cudaError_t e = launch_sample(j, c->img.W, cfg, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "sample kernel launch");
    return KSIM_OK;
}

ksim_status ksim_component_sample(ksim_component *c, const uint8_t *f_sel, int64_t B, uint64_t seed,
                                  int32_t rng_mode, uint8_t *out)
{
    if (!c) return fail(KSIM_ERR_INVALID_ARGUMENT, "component is NULL");
    if (B < 0) return fail(KSIM_ERR_INVALID_ARGUMENT, "B must be >= 0");
    if (check_rng(rng_mode) != KSIM_OK) return KSIM_ERR_INVALID_ARGUMENT;
    const int F = c->img.F, n_out = c->img.n_out;
    if (B == 0) return KSIM_OK;
    if ((F > 0 && !f_sel) || !out) return fail(KSIM_ERR_INVALID_ARGUMENT, "input or output pointer is NULL");
    if (n_out == 0) {  // the reference pads its output to one zero column (kokkos_sim.cpp:233-240)
        std::memset(out, 0, (size_t)B);
        return KSIM_OK;
    }
    // the pipelined host call of the component alone as a program: identity
    // f_selection and output order, component seed offset 0, so the bits are
    // this component's
    ksim_program *p = nullptr;
    {
        DeviceGuard g(c->device);
        std::lock_guard<std::mutex> lk(c->mu);
        if (!c->self_prog) {
            std::vector<int32_t> sel((size_t)F), order((size_t)n_out);
            std::iota(sel.begin(), sel.end(), 0);
            std::iota(order.begin(), order.end(), 0);
            ksim_component *comps[1] = {c};
            const int32_t *sels[1] = {sel.data()};
            const int32_t lens[1] = {F};
            const ksim_status st = ksim_program_create(comps, 1, sels, lens, order.data(), n_out, &c->self_prog);
            if (st != KSIM_OK) return st;
        }
        p = c->self_prog;
    }
    return program_sample_host(p, f_sel, B, F, seed, rng_mode, out, false);
}

static ksim_status eval_common(ksim_component *c, int32_t graph, const uint8_t *params, int64_t B, int64_t P,
                               int mode, void *out, size_t out_bytes)
{
    if (!c) return fail(KSIM_ERR_INVALID_ARGUMENT, "component is NULL");
    if (graph < 0 || graph >= c->img.n_graphs)
        return fail(KSIM_ERR_INVALID_ARGUMENT, "graph index out of range");
    if (B < 0 || P < 0) return fail(KSIM_ERR_INVALID_ARGUMENT, "B and P must be >= 0");
    if (B == 0) return KSIM_OK;
    if ((P > 0 && !params) || !out) return fail(KSIM_ERR_INVALID_ARGUMENT, "input or output pointer is NULL");
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    cudaError_t e = c->ws_f.ensure((size_t)std::max<int64_t>(B * P, 1));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(params workspace)");
    e = c->ws_aux.ensure(out_bytes);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(eval output)");
    if (P > 0) {
        e = cudaMemcpyAsync(c->ws_f.p, params, (size_t)(B * P), cudaMemcpyHostToDevice, c->stream);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(params)");
    }
    EvalJob j = {};
    j.image = c->d_image;
    j.gdir = (const GraphDir *)c->d_image;
    j.graph = graph;
    j.params = (const uint8_t *)c->ws_f.p;
    j.B = B;
    j.P = P;
    j.mode = mode;
    j.out = c->ws_aux.p;
    j.status = c->d_status;
    e = launch_eval(j, c->img.W, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "eval kernel launch");
    e = cudaMemcpyAsync(out, c->ws_aux.p, out_bytes, cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(eval out)");
    e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "eval");
    return KSIM_OK;
}

ksim_status ksim_component_eval_abs(ksim_component *c, int32_t graph, const uint8_t *params, int64_t B,
                                    int64_t P, double *out)
{
    return eval_common(c, graph, params, B, P, EVAL_ABS, out, (size_t)std::max<int64_t>(B, 0) * 8);
}

ksim_status ksim_component_eval(ksim_component *c, int32_t graph, const uint8_t *params, int64_t B, int64_t P,
                                double *out_re_im)
{
    return eval_common(c, graph, params, B, P, EVAL_COMPLEX, out_re_im, (size_t)std::max<int64_t>(B, 0) * 16);
}

ksim_status ksim_component_eval_terms(ksim_component *c, int32_t graph, const uint8_t *params, int64_t B,
                                      int64_t P, int64_t *out)
{
    if (!c || graph < 0 || graph >= c->img.n_graphs)
        return fail(KSIM_ERR_INVALID_ARGUMENT, "component is NULL or graph index out of range");
    const int64_t G = c->img.gdir[graph].G;
    if (G == 0) return KSIM_OK;
    return eval_common(c, graph, params, B, P, EVAL_TERMS, out, (size_t)std::max<int64_t>(B, 0) * G * 40);
}

ksim_status ksim_component_status(ksim_component *c, uint32_t *flags, int32_t reset)
{
    if (!c || !flags) return fail(KSIM_ERR_INVALID_ARGUMENT, "component or flags is NULL");
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess) e = cudaMemcpy(flags, c->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && reset) e = cudaMemset(c->d_status, 0, sizeof(uint32_t));
    if (e != cudaSuccess) return cuda_fail(e, "status");
    return KSIM_OK;
}

// ---- program ---------------------------------------------------------------

ksim_status ksim_program_create(ksim_component *const *comps, int32_t n_comps, const int32_t *const *f_selection,
                                const int32_t *f_sel_len, const int32_t *output_order, int32_t n_outputs,
                                ksim_program **out)
{
    if (!out) return fail(KSIM_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (n_comps < 0 || n_outputs < 0 || (n_comps > 0 && (!comps || !f_selection || !f_sel_len)) ||
        (n_outputs > 0 && !output_order))
        return fail(KSIM_ERR_INVALID_ARGUMENT, "bad program arguments");
    int total = 0;
    int device = -1;
    for (int k = 0; k < n_comps; ++k) {
        if (!comps[k]) return fail(KSIM_ERR_INVALID_ARGUMENT, "component is NULL");
        if (f_sel_len[k] != comps[k]->img.F)
            return fail(KSIM_ERR_INVALID_ARGUMENT, "component " + std::to_string(k) +
                                                       ": f_selection length != num_f");
        if (device >= 0 && comps[k]->device != device)
            return fail(KSIM_ERR_INVALID_ARGUMENT, "components live on different devices");
        device = comps[k]->device;
        total += comps[k]->img.n_out;
    }
    if (total != n_outputs)
        return fail(KSIM_ERR_INVALID_ARGUMENT, "len(output_order) != total outputs of the components");
    // combined column c goes to output column j with argsort(output_order)[j] == c
    std::vector<int> perm(n_outputs);
    for (int i = 0; i < n_outputs; ++i) perm[i] = i;
    std::stable_sort(perm.begin(), perm.end(),
                     [&](int a, int b) { return output_order[a] < output_order[b]; });
    for (int i = 1; i < n_outputs; ++i)
        if (output_order[perm[i]] == output_order[perm[i - 1]])
            return fail(KSIM_ERR_INVALID_ARGUMENT, "output_order has duplicate values");
    std::vector<int32_t> dest(n_outputs);
    for (int j2 = 0; j2 < n_outputs; ++j2) dest[perm[j2]] = j2;

    std::unique_ptr<ksim_program> p(new ksim_program());
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) return fail(KSIM_ERR_NO_DEVICE, "cudaGetDevice");
    p->device = device;
    p->n_outputs = n_outputs;
    DeviceGuard g(device);
    int off = 0;
    for (int k = 0; k < n_comps; ++k) {
        ksim_component *c = comps[k];
        ProgramPart part;
        part.comp = c;
        const int F = c->img.F;
        for (int jx = 0; jx < F; ++jx) {
            if (f_selection[k][jx] < 0)
                return fail(KSIM_ERR_INVALID_ARGUMENT, "negative f_selection entry");
            p->min_f_cols = std::max(p->min_f_cols, f_selection[k][jx] + 1);
        }
        cudaError_t e = cudaMalloc(&part.d_sel, sizeof(int32_t) * std::max(F, 1));
        if (e == cudaSuccess && F > 0)
            e = cudaMemcpy(part.d_sel, f_selection[k], sizeof(int32_t) * F, cudaMemcpyHostToDevice);
        const int n = c->img.n_out;
        if (e == cudaSuccess) e = cudaMalloc(&part.d_cols, sizeof(int32_t) * std::max(n, 1));
        if (e == cudaSuccess && n > 0)
            e = cudaMemcpy(part.d_cols, dest.data() + off, sizeof(int32_t) * n, cudaMemcpyHostToDevice);
        p->parts.push_back(part);
        if (e != cudaSuccess) {
            ksim_program_destroy(p.release());
            return cuda_fail(e, "program upload");
        }
        off += n;
    }
    std::vector<cudaStream_t *> streams = {&p->s_h2d, &p->s_d2h};
    for (cudaStream_t &st : p->cs) streams.push_back(&st);
    for (cudaStream_t *st : streams) {
        cudaError_t e = cudaStreamCreateWithFlags(st, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            ksim_program_destroy(p.release());
            return cuda_fail(e, "cudaStreamCreate");
        }
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device);
    p->wave_shots = (int64_t)std::max(sms, 1) * 5 * 256;  // five CTAs of 256 shots per SM
    cudaError_t e = cudaMallocHost(&p->h_status, sizeof(uint32_t) * std::max<size_t>(p->parts.size(), 1));
    if (e != cudaSuccess) {
        ksim_program_destroy(p.release());
        return cuda_fail(e, "cudaMallocHost(status words)");
    }
    *out = p.release();
    return KSIM_OK;
}

void ksim_program_destroy(ksim_program *p)
{
    if (!p) return;
    DeviceGuard g(p->device);
    std::vector<cudaStream_t> streams = {p->s_h2d, p->s_d2h};
    for (cudaStream_t st : p->cs) streams.push_back(st);
    for (cudaStream_t st : streams)
        if (st) cudaStreamSynchronize(st);
    for (auto &part : p->parts) {
        if (part.d_sel) cudaFree(part.d_sel);
        if (part.d_cols) cudaFree(part.d_cols);
    }
    p->ws_f.release();
    p->ws_out.release();
    p->ws_fp.release();
    p->ws_op.release();
    for (cudaStream_t st : streams)
        if (st) cudaStreamDestroy(st);
    for (cudaEvent_t ev : p->ev_in) cudaEventDestroy(ev);
    for (cudaEvent_t ev : p->ev_done) cudaEventDestroy(ev);
    if (p->h_status) cudaFreeHost(p->h_status);
    delete p;
}

int32_t ksim_program_n_outputs(const ksim_program *p) { return p ? p->n_outputs : -1; }
int32_t ksim_program_n_components(const ksim_program *p) { return p ? (int32_t)p->parts.size() : -1; }

ksim_status ksim_program_job(const ksim_program *p, int32_t k, const uint8_t *d_f, int64_t f_stride, uint8_t *d_out,
                             int64_t B, int64_t shot_offset, uint64_t seed, int32_t rng_mode, ksim_batch_job *out)
{
    if (!p || !out || k < 0 || k >= (int32_t)p->parts.size())
        return fail(KSIM_ERR_INVALID_ARGUMENT, "bad program / component index");
    if (f_stride < p->min_f_cols) return fail(KSIM_ERR_INVALID_ARGUMENT, "f_stride below the f_selection width");
    const ProgramPart &part = p->parts[k];
    ksim_batch_job j = {};
    j.comp = part.comp;
    j.d_f = d_f;
    j.f_stride = f_stride;
    j.d_f_sel = part.d_sel;
    j.d_out = d_out;
    j.out_stride = p->n_outputs;
    j.out_col0 = 0;
    j.d_out_cols = part.d_cols;
    j.B = B;
    j.shot_offset = shot_offset;
    j.seed = seed + 0x9E37ull * (uint64_t)k;
    j.rng_mode = rng_mode;
    *out = j;
    return KSIM_OK;
}
int32_t ksim_program_min_f_cols(const ksim_program *p) { return p ? p->min_f_cols : -1; }

ksim_status ksim_program_sample_device(ksim_program *p, const uint8_t *d_f_params, int64_t B, int64_t n_f_cols,
                                       int64_t shot_offset, uint64_t seed, int32_t rng_mode, uint8_t *d_out,
                                       void *stream)
{
    if (!p) return fail(KSIM_ERR_INVALID_ARGUMENT, "program is NULL");
    if (B < 0 || shot_offset < 0) return fail(KSIM_ERR_INVALID_ARGUMENT, "B and shot_offset must be >= 0");
    if (check_rng(rng_mode) != KSIM_OK) return KSIM_ERR_INVALID_ARGUMENT;
    if (n_f_cols < p->min_f_cols)
        return fail(KSIM_ERR_INVALID_ARGUMENT, "f_params has " + std::to_string(n_f_cols) +
                                                   " columns; f_selection needs " +
                                                   std::to_string(p->min_f_cols));
    if (B == 0 || p->n_outputs == 0) return KSIM_OK;
    if ((n_f_cols > 0 && !d_f_params) || !d_out) return fail(KSIM_ERR_INVALID_ARGUMENT, "NULL buffer");
    DeviceGuard g(p->device);
    for (size_t k = 0; k < p->parts.size(); ++k) {
        ksim_component *c = p->parts[k].comp;
        if (c->img.n_out == 0) continue;
        LaunchCfg cfg;
        {
            std::lock_guard<std::mutex> lk(c->mu);
            cfg = c->cfg;
        }
        SampleJob j = {};
        ksim_status st = component_job(c, cfg, j);
        if (st != KSIM_OK) return st;
        j.rng_mode = rng_mode;
        j.f = d_f_params;
        j.f_stride = n_f_cols;
        j.f_sel = p->parts[k].d_sel;
        j.out = d_out;
        j.out_stride = p->n_outputs;
        j.out_cols = p->parts[k].d_cols;
        j.B = B;
        j.shot_offset = shot_offset;
        j.seed = seed + 0x9E37ull * (uint64_t)k;
        cudaError_t e = launch_sample(j, c->img.W, cfg, (cudaStream_t)stream);
        if (e != cudaSuccess) return cuda_fail(e, "sample kernel launch");
    }
    return KSIM_OK;
}

}  // extern "C"

namespace {

// Host buffers in, host buffers out, in chunks of shots (host_chunk_bounds)
// pipelined over copy and compute streams: the f rows of chunk i+1 cross
// PCIe while chunk i samples, the results of chunk i cross back while later
// chunks sample (page-locked buffers), and consecutive chunks take the
// compute streams in turn so their waves of CTAs overlap.  Chunk c samples with shot_offset = its first
// row, so the bits equal a single launch over all B shots.
// packed: f rows of ceil(n_f_cols/8) bytes and output rows of
// ceil(n_outputs/8) bytes, bit c of a row in byte c/8 at bit c%8.
// noise (nullable): f rows are drawn on the device from this model with
// noise_seed instead of being copied from `f`.
ksim_status program_sample_host(ksim_program *p, const uint8_t *f, int64_t B, int64_t n_f_cols, uint64_t seed,
                                int32_t rng_mode, uint8_t *out, bool packed, const ksim_noise *noise,
                                uint64_t noise_seed)
{
    if (!p) return fail(KSIM_ERR_INVALID_ARGUMENT, "program is NULL");
    if (B < 0 || n_f_cols < 0) return fail(KSIM_ERR_INVALID_ARGUMENT, "B and n_f_cols must be >= 0");
    if (B == 0 || p->n_outputs == 0) return check_rng(rng_mode);
    if ((n_f_cols > 0 && !f && !noise) || !out) return fail(KSIM_ERR_INVALID_ARGUMENT, "NULL buffer");
    if (check_rng(rng_mode) != KSIM_OK) return KSIM_ERR_INVALID_ARGUMENT;
    if (n_f_cols < p->min_f_cols)
        return fail(KSIM_ERR_INVALID_ARGUMENT, "f_params has " + std::to_string(n_f_cols) +
                                                   " columns; f_selection needs " + std::to_string(p->min_f_cols));
    DeviceGuard g(p->device);
    std::lock_guard<std::mutex> lk(p->mu);
    const int64_t n_out = p->n_outputs;
    const int64_t f_row = packed ? (n_f_cols + 7) / 8 : n_f_cols;
    const int64_t o_row = packed ? (n_out + 7) / 8 : n_out;
    cudaError_t e = p->ws_f.ensure((size_t)std::max<int64_t>(B * n_f_cols, 1));
    if (e == cudaSuccess) e = p->ws_out.ensure((size_t)(B * n_out));
    if (e == cudaSuccess && packed) e = p->ws_fp.ensure((size_t)std::max<int64_t>(B * f_row, 1));
    if (e == cudaSuccess && packed) e = p->ws_op.ensure((size_t)(B * o_row));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(program workspace)");
    uint8_t *d_f = (uint8_t *)p->ws_f.p, *d_out = (uint8_t *)p->ws_out.p;
    uint8_t *d_in = packed ? (uint8_t *)p->ws_fp.p : d_f;       // where the host rows land
    uint8_t *d_back = packed ? (uint8_t *)p->ws_op.p : d_out;   // what goes back

    const std::vector<int64_t> bounds = host_chunk_bounds(B, (noise ? 0 : f_row) + o_row);
    const int n_chunks = (int)bounds.size() - 1;
    const int lag = host_copy_lag(bounds, p->wave_shots, KSIM_HOST_STREAMS);
    std::vector<cudaEvent_t> &ev_in = p->ev_in, &ev_done = p->ev_done;
    ksim_status st = KSIM_OK;
    while ((int)ev_in.size() < n_chunks && e == cudaSuccess) {
        cudaEvent_t a = nullptr, b = nullptr;
        e = cudaEventCreateWithFlags(&a, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            if (a) cudaEventDestroy(a);
            break;
        }
        ev_in.push_back(a);
        ev_done.push_back(b);
    }
    auto copy_back = [&](int i) -> cudaError_t {
        const int64_t c0 = bounds[i], n = bounds[i + 1] - c0;
        cudaError_t x = cudaStreamWaitEvent(p->s_d2h, ev_done[i], 0);
        if (x == cudaSuccess)
            x = cudaMemcpyAsync(out + c0 * o_row, d_back + c0 * o_row, (size_t)(n * o_row), cudaMemcpyDeviceToHost,
                                p->s_d2h);
        return x;
    };
    for (int i = 0; i < n_chunks && e == cudaSuccess && st == KSIM_OK; ++i) {
        const int64_t c0 = bounds[i], n = bounds[i + 1] - c0;
        cudaStream_t cs = p->cs[i % KSIM_HOST_STREAMS];
        if (noise) {
            e = launch_noise(noise, n, c0, noise_seed, d_f + c0 * n_f_cols, n_f_cols, cs);
        } else {
            if (f_row > 0)
                e = cudaMemcpyAsync(d_in + c0 * f_row, f + c0 * f_row, (size_t)(n * f_row), cudaMemcpyHostToDevice,
                                    p->s_h2d);
            if (e == cudaSuccess) e = cudaEventRecord(ev_in[i], p->s_h2d);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, ev_in[i], 0);
        }
        if (e == cudaSuccess && packed)
            e = launch_unpack_bits(d_in + c0 * f_row, n, f_row, n_f_cols, d_f + c0 * n_f_cols, cs);
        if (e != cudaSuccess) break;
        st = ksim_program_sample_device(p, d_f + c0 * n_f_cols, n, n_f_cols, c0, seed, rng_mode, d_out + c0 * n_out,
                                        cs);
        if (st != KSIM_OK) break;
        if (packed) e = launch_pack_bits(d_out + c0 * n_out, n, n_out, o_row, d_back + c0 * o_row, cs);
        if (e == cudaSuccess) e = cudaEventRecord(ev_done[i], cs);
        // chunk i - lag's output copy once chunk i is queued: into
        // page-locked memory copies are asynchronous and start as each chunk
        // ends; into pageable memory each one holds the host until it is
        // done, so the lag keeps about a wave of CTAs queued meanwhile (small
        // chunks: up to one per compute stream) without leaving more than
        // that many copies for after the last chunk
        if (e == cudaSuccess && i >= lag) e = copy_back(i - lag);
    }
    for (int i = std::max(0, n_chunks - lag); i < n_chunks && e == cudaSuccess && st == KSIM_OK; ++i)
        e = copy_back(i);
    // the components' status words behind the last output copy (the output
    // stream has waited for every chunk's sampling by then)
    for (size_t k = 0; k < p->parts.size() && e == cudaSuccess && st == KSIM_OK; ++k)
        e = cudaMemcpyAsync(p->h_status + k, p->parts[k].comp->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                            p->s_d2h);
    if (e == cudaSuccess && st == KSIM_OK) {
        // every chunk's output copy waited for its sampling, which waited for
        // its input copy: the output stream's end is the call's end
        e = cudaStreamSynchronize(p->s_d2h);
    } else {
        std::vector<cudaStream_t> streams = {p->s_h2d, p->s_d2h};
        for (cudaStream_t x : p->cs) streams.push_back(x);
        for (cudaStream_t x : streams) cudaStreamSynchronize(x);
    }
    if (st != KSIM_OK) return st;
    if (e != cudaSuccess) return cuda_fail(e, "program sample");
    ksim_status rep = KSIM_OK;
    for (size_t k = 0; k < p->parts.size(); ++k) {
        const ksim_status r = report_timeout_flags(p->parts[k].comp, p->h_status[k]);
        if (rep == KSIM_OK) rep = r;
    }
    return rep;
}

}  // namespace

extern "C" {

ksim_status ksim_program_sample(ksim_program *p, const uint8_t *f_params, int64_t B, int64_t n_f_cols,
                                uint64_t seed, int32_t rng_mode, uint8_t *out)
{
    return program_sample_host(p, f_params, B, n_f_cols, seed, rng_mode, out, false);
}

ksim_status ksim_program_sample_packed(ksim_program *p, const uint8_t *f_packed, int64_t B, int64_t n_f_cols,
                                       uint64_t seed, int32_t rng_mode, uint8_t *out_packed)
{
    return program_sample_host(p, f_packed, B, n_f_cols, seed, rng_mode, out_packed, true);
}

ksim_status ksim_program_sample_noisy(ksim_program *p, ksim_noise *n, int64_t B, uint64_t noise_seed, uint64_t seed,
                                      int32_t rng_mode, uint8_t *out)
{
    if (!p || !n) return fail(KSIM_ERR_INVALID_ARGUMENT, "program or noise model is NULL");
    if (noise_device(n) != p->device)
        return fail(KSIM_ERR_INVALID_ARGUMENT, "program and noise model live on different devices");
    if (ksim_noise_num_f(n) < p->min_f_cols)
        return fail(KSIM_ERR_INVALID_ARGUMENT, "the noise model draws " + std::to_string(ksim_noise_num_f(n)) +
                                                   " f parameters; f_selection needs " +
                                                   std::to_string(p->min_f_cols));
    return program_sample_host(p, nullptr, B, ksim_noise_num_f(n), seed, rng_mode, out, false, n, noise_seed);
}

}  // extern "C"
