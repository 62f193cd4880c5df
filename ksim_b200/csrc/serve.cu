// serve.cu — continuous-batching sampling server with a device-resident loop.
//
// Device side (k_serve): a persistent grid drains a ring of jobs (one job =
// one component of one admitted request) tile by tile.  Thread 0 of a CTA
// claims the next tile of the job at the ring head with one atomicAdd; when
// the head job has no tiles left it advances the head with a CAS and tries
// the next, so the tiles of every request admitted so far are handed out in
// arrival order while earlier requests are still running on other CTAs.  The
// CTA copies the job's descriptor into shared memory with L2-only loads and
// runs the sampling tile (sample_tile.cuh, L2-coherent loads, one staging
// ring per CTA for its whole life).  The CTA that finishes a job's last tile
// decrements the request's job count; the one that finishes the request
// writes the request's sequence number into a host-mapped flag after a
// system-scope fence.  With nothing to claim, thread 0 backs off with
// __nanosleep.  Leaving is collective: a CTA gives up only when no CTA of
// the grid has claimed a tile for idle_us (the claim time is shared in the
// control block), and the first to give up raises an exit word that makes
// every other CTA leave at its next claim, so the grid never shrinks while
// the kernel runs; the scheduler relaunches a full grid when work arrives.
// Every wait in the loop is bounded.
//
// Host side (ksim_server): submit() queues a request; one scheduler thread
//   1. admits queued requests in arrival order by HBM footprint
//      (serve_sched.h): f rows and output rows get an arena block, the f rows
//      are copied in (cudaMemcpy2DAsync), then the job descriptors, the
//      request record and the ring entries, all in order on one copy stream,
//      so the loop can only see a ring entry whose data is in place;
//   2. (re)launches the loop kernel whenever work is in flight and no loop is
//      running;
//   3. polls the completion flags, copies finished outputs (and the request's
//      status word) to the caller's buffer on a second copy stream, and frees
//      the request's resources once that copy is done.
// Programs with parameter vectors wider than 256 bits (W > 4) are not in the
// loop kernel's instantiations; their requests run as plain launches on a
// side stream, admitted and completed through the same queue.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ksim_b200.h"
#include "kernels.h"
#include "runtime.h"
#include "sample_tile.cuh"
#include "serve_sched.h"

namespace ksim {

struct ServeJob {
    SampleJob j;
    int32_t W, n_tiles;
    int32_t next_tile;  // tiles handed out (atomic)
    int32_t remaining;  // tiles not finished (atomic)
    int32_t req_slot, paths;  // paths: the component's term paths (LaunchCfg::paths)
    int64_t pad1;
};
static_assert(sizeof(SampleJob) % 16 == 0, "SampleJob is copied in 16-byte words");
static_assert(sizeof(ServeJob) % 16 == 0, "ServeJob table entries stay 16-byte aligned");

struct ServeReqDev {
    int32_t remaining_jobs;  // atomic
    uint32_t seq;            // written to the host flag when the request is done
    uint32_t flags;          // KSIM_FLAG_* of the request's jobs
    uint32_t pad;
};

struct ServeCtl {
    unsigned long long head;  // ring position of the first job that may have tiles left
    long long last_claim_ns;  // globaltimer of the latest tile claim of any CTA
    int32_t stop;             // set by the host at shutdown
    int32_t exiting;          // set by the first CTA that leaves; cleared before each launch
};

namespace {

constexpr int SERVE_SCAN = 64;           // ring positions a claim looks at before backing off
constexpr unsigned SERVE_SLEEP_MAX = 8192;  // ns

__device__ __forceinline__ long long global_ns()
{
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <typename T>
__device__ __forceinline__ T vload(const T *p)
{
    return *(const volatile T *)p;
}

// One tile of a job with the body compiled for the job's W and term paths.
// The loop inlines the bodies that carry most requests (all-32-bit W = 1
// and 2, 32-bit and hybrid W = 2) and calls the others out of line (a call
// costs the body about a tenth of its speed; inlining every body would
// bloat the loop).  Job data comes through L2-only loads (CG): buffers are
// reused across requests within one kernel lifetime.
template <int W, int PATHS>
__device__ __noinline__ bool serve_tile(const SampleJob &j, int64_t s0, uint64_t *bar, uint8_t *slots, uint32_t &g,
                                        uint8_t *scratch)
{
    return sample_tile<W, true, true, shots_per_thread(W), PATHS>(j, s0, bar, slots, g, scratch);
}

__global__ void __launch_bounds__(256, KSIM_SAMPLE_MIN_CTAS) k_serve(ServeJob *jobs, ServeReqDev *reqs, const unsigned long long *ring,
                                               int ring_cap, ServeCtl *ctl, uint32_t *done_flags, long long idle_ns)
{
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(16) SampleJob s_job;
    __shared__ int s_slot, s_tile, s_W, s_paths;
    uint64_t *bar = (uint64_t *)smem;
    uint8_t *slots = smem + BAR_BYTES;
    ring_init(bar);
    uint32_t g = 0;
    const long long t_start = global_ns();
    unsigned backoff = 64;
    for (;;) {
        if (threadIdx.x == 0) {
            int slot = -1, tile = -1;
            for (int scan = 0; scan < SERVE_SCAN && !vload(&ctl->exiting); ++scan) {
                const unsigned long long h = vload(&ctl->head);
                const unsigned long long e = vload(ring + (h % (unsigned long long)ring_cap));
                if ((uint32_t)(e >> 32) != (uint32_t)(h + 1)) break;  // not published yet
                const int js = (int)(uint32_t)e;
                const int t = atomicAdd(&jobs[js].next_tile, 1);
                if (t < vload(&jobs[js].n_tiles)) {
                    slot = js;
                    tile = t;
                    break;
                }
                atomicCAS(&ctl->head, h, h + 1);  // exhausted: move the head on
            }
            if (slot >= 0) {
                backoff = 64;
                *(volatile long long *)&ctl->last_claim_ns = global_ns();
                s_W = vload(&jobs[slot].W);
                s_paths = vload(&jobs[slot].paths);
            } else {
                const long long now = global_ns();
                const long long last = vload(&ctl->last_claim_ns);
                const long long ref = last > t_start ? last : t_start;
                if (vload(&ctl->exiting) || vload(&ctl->stop) || now - ref > idle_ns) {
                    atomicExch(&ctl->exiting, 1);
                    slot = -2;
                } else {
                    __nanosleep(backoff);
                    backoff = backoff * 2 > SERVE_SLEEP_MAX ? SERVE_SLEEP_MAX : backoff * 2;
                }
            }
            s_slot = slot;
            s_tile = tile;
        }
        __syncthreads();
        const int slot = s_slot;
        if (slot == -2) break;
        if (slot >= 0) {
            constexpr int NW = (int)(sizeof(SampleJob) / 16);
            if (threadIdx.x < NW)
                ((int4 *)&s_job)[threadIdx.x] = __ldcg((const int4 *)&jobs[slot].j + threadIdx.x);
        }
        __syncthreads();
        if (slot >= 0) {
            constexpr int S = shots_per_thread(4);  // every loop job has W <= 4
            const int64_t s0 = (int64_t)s_tile * blockDim.x * S;
            uint8_t *scratch = slots + (size_t)NSLOT * s_job.slot_bytes;
            bool ok;
            const int paths = s_paths;
#define KSIM_SERVE_W(WW)                                                                                \
    case WW:                                                                                            \
        ok = paths == PATHS_NARROW ? serve_tile<WW, PATHS_NARROW>(s_job, s0, bar, slots, g, scratch)    \
             : paths == PATHS_NARROW_HYBRID                                                             \
                 ? serve_tile<WW, PATHS_NARROW_HYBRID>(s_job, s0, bar, slots, g, scratch)              \
                 : serve_tile<WW, PATHS_ALL>(s_job, s0, bar, slots, g, scratch);                       \
        break;
            // the common bodies inline, the rest out of line
            if (s_W == 1 && paths == PATHS_NARROW)
                ok = sample_tile<1, true, true, shots_per_thread(1), PATHS_NARROW>(s_job, s0, bar, slots, g, scratch);
            else if (s_W == 2 && paths == PATHS_NARROW)
                ok = sample_tile<2, true, true, shots_per_thread(2), PATHS_NARROW>(s_job, s0, bar, slots, g, scratch);
            else if (s_W == 2 && paths == PATHS_NARROW_HYBRID)
                ok = sample_tile<2, true, true, shots_per_thread(2), PATHS_NARROW_HYBRID>(s_job, s0, bar, slots, g, scratch);
            else {
            switch (s_W) {
            KSIM_SERVE_W(1) KSIM_SERVE_W(2) KSIM_SERVE_W(3)
            default: KSIM_SERVE_W(4)
            }
            }
#undef KSIM_SERVE_W
            __threadfence();  // this thread's outputs before the counters below
            __syncthreads();
            if (threadIdx.x == 0) {
                if (atomicSub(&jobs[slot].remaining, 1) == 1) {
                    const int rs = vload(&jobs[slot].req_slot);
                    __threadfence();
                    if (atomicSub(&reqs[rs].remaining_jobs, 1) == 1) {
                        const uint32_t seq = vload(&reqs[rs].seq);
                        __threadfence_system();
                        *(volatile uint32_t *)&done_flags[rs] = seq;
                    }
                }
            }
            if (!ok) break;  // a staging wait ran out: this CTA's ring is out of phase
        }
        __syncthreads();  // s_* are rewritten by the next claim
    }
}

using Clock = std::chrono::steady_clock;

double to_seconds(Clock::time_point t)
{
    return std::chrono::duration<double>(t.time_since_epoch()).count();
}

enum ReqState { R_PENDING = 0, R_RUNNING = 1, R_COPYING = 2, R_DONE = 3 };

struct ServeRequest {
    int64_t id = 0;
    ksim_program *prog = nullptr;
    const uint8_t *f = nullptr;
    uint8_t *out = nullptr;
    int64_t B = 0, n_f_cols = 0, f_stride = 0, f_bytes = 0, out_bytes = 0;
    uint64_t seed = 0;
    int32_t rng_mode = 0;
    int n_jobs = 0;
    bool loop = true;
    int64_t arena_off = -1;
    int slot = -1;
    uint32_t seq = 0;
    std::vector<int> jobs;
    int state = R_PENDING;
    ksim_status status = KSIM_OK;
    std::string error;
    cudaEvent_t ev = nullptr;  // side launch done (R_RUNNING) / output copy done (R_COPYING)
    Clock::time_point t_submit, t_done;
};

}  // namespace
}  // namespace ksim

using namespace ksim;

struct ksim_server {
    int device = 0;
    ksim_server_config cfg = {};
    LaunchCfg lcfg;
    int grid = 0;
    size_t smem = 0;

    uint8_t *d_arena = nullptr;
    Arena arena;
    SlotPool req_slots, job_slots;
    ServeJob *d_jobs = nullptr, *h_jobs = nullptr;
    ServeReqDev *d_reqs = nullptr, *h_reqs = nullptr, *h_reqs_back = nullptr;
    unsigned long long *d_ring = nullptr, *h_ring = nullptr;
    int ring_cap = 0;
    unsigned long long ring_tail = 0;
    int64_t jobs_in_flight = 0;
    ServeCtl *d_ctl = nullptr;
    uint32_t *h_done = nullptr, *d_done = nullptr;
    int32_t *h_stop = nullptr;

    cudaStream_t s_h2d = nullptr, s_d2h = nullptr, s_loop = nullptr, s_side = nullptr;
    cudaEvent_t loop_done = nullptr, h2d_mark = nullptr;
    bool loop_running = false;

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread worker;
    bool stopping = false;
    std::deque<ServeRequest *> pending;
    std::vector<ServeRequest *> running;  // admitted, not finished
    std::map<int64_t, std::unique_ptr<ServeRequest>> all;
    int64_t next_id = 1;
    uint32_t next_seq = 1;
    ksim_server_stats st = {};
    std::string fatal;  // a CUDA failure of the scheduler (every later request fails with it)
};

namespace ksim {
namespace {

void finish(ksim_server *s, ServeRequest *r, ksim_status status, const std::string &err)
{
    r->state = R_DONE;
    r->status = status;
    r->error = err;
    r->t_done = Clock::now();
    if (status == KSIM_OK) {
        s->st.completed += 1;
        s->st.shots_completed += r->B;
    } else if (status == KSIM_ERR_CANCELLED) {
        s->st.cancelled += 1;
    } else {
        s->st.failed += 1;
    }
}

// Release an admitted request's device resources (caller holds mu).
void release(ksim_server *s, ServeRequest *r)
{
    if (r->arena_off >= 0) s->arena.release(r->arena_off);
    r->arena_off = -1;
    for (int j : r->jobs) s->job_slots.give(j);
    s->jobs_in_flight -= (int64_t)r->jobs.size();
    r->jobs.clear();
    if (r->slot >= 0) s->req_slots.give(r->slot);
    r->slot = -1;
    if (r->ev) cudaEventDestroy(r->ev);
    r->ev = nullptr;
}

int words_of(const ksim_program *p)
{
    int w = 1;
    for (const ProgramPart &part : p->parts) w = std::max(w, part.comp->img.W);
    return w;
}

// Admit and publish one request (caller holds mu; resources were checked).
ksim_status admit(ksim_server *s, ServeRequest *r)
{
    ksim_program *p = r->prog;
    const int64_t f_region = Arena::round_up(std::max<int64_t>(r->f_bytes, 1), 256);
    r->arena_off = s->arena.alloc(f_region + std::max<int64_t>(r->out_bytes, 1));
    if (r->arena_off < 0) return fail(KSIM_ERR_INTERNAL, "arena block vanished between check and admit");
    r->slot = s->req_slots.take();
    r->seq = s->next_seq++;
    if (s->next_seq == 0) s->next_seq = 1;
    uint8_t *d_f = s->d_arena + r->arena_off;
    uint8_t *d_out = d_f + f_region;
    cudaError_t e = cudaSuccess;
    if (r->f_bytes > 0)
        e = cudaMemcpy2DAsync(d_f, (size_t)r->n_f_cols, r->f, (size_t)r->f_stride, (size_t)r->n_f_cols, (size_t)r->B,
                              cudaMemcpyHostToDevice, s->s_h2d);
    if (e != cudaSuccess) return cuda_fail(e, "server: f copy");
    if (!r->loop) {
        // plain launches on the side stream, after the f copy
        e = cudaEventRecord(s->h2d_mark, s->s_h2d);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s->s_side, s->h2d_mark, 0);
        if (e != cudaSuccess) return cuda_fail(e, "server: side ordering");
        ksim_status st = ksim_program_sample_device(p, d_f, r->B, r->n_f_cols, 0, r->seed, r->rng_mode, d_out,
                                                    s->s_side);
        if (st != KSIM_OK) return st;
        e = cudaEventCreateWithFlags(&r->ev, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(r->ev, s->s_side);
        if (e != cudaSuccess) return cuda_fail(e, "server: side event");
        s->st.side_launches += 1;
        r->state = R_RUNNING;
        return KSIM_OK;
    }
    // job descriptors
    const int64_t tile = (int64_t)s->lcfg.threads * shots_per_thread(4);
    const int64_t tiles = (r->B + tile - 1) / tile;
    std::vector<int> new_jobs;
    for (size_t k = 0; k < p->parts.size(); ++k) {
        ksim_component *c = p->parts[k].comp;
        if (c->img.n_out == 0) continue;
        const int js = s->job_slots.take();
        new_jobs.push_back(js);
        r->jobs.push_back(js);
        s->jobs_in_flight += 1;
        ServeJob &J = s->h_jobs[js];
        J = ServeJob();
        ksim_status st = component_job(c, s->lcfg, J.j);
        if (st != KSIM_OK) return st;
        J.j.rng_mode = r->rng_mode;
        J.j.f = d_f;
        J.j.f_stride = r->n_f_cols;
        J.j.f_sel = p->parts[k].d_sel;
        J.j.out = d_out;
        J.j.out_stride = p->n_outputs;
        J.j.out_col0 = 0;
        J.j.out_cols = p->parts[k].d_cols;
        J.j.amp = nullptr;
        J.j.B = r->B;
        J.j.shot_offset = 0;
        J.j.seed = r->seed + 0x9E37ull * (uint64_t)k;
        J.j.status = &s->d_reqs[r->slot].flags;
        J.W = c->img.W;
        J.paths = c->cfg.paths;
        J.n_tiles = (int32_t)tiles;
        J.next_tile = 0;
        J.remaining = (int32_t)tiles;
        J.req_slot = r->slot;
        e = cudaMemcpyAsync(&s->d_jobs[js], &J, sizeof(ServeJob), cudaMemcpyHostToDevice, s->s_h2d);
        if (e != cudaSuccess) return cuda_fail(e, "server: job copy");
    }
    ServeReqDev &R = s->h_reqs[r->slot];
    R.remaining_jobs = (int32_t)new_jobs.size();
    R.seq = r->seq;
    R.flags = 0;
    R.pad = 0;
    e = cudaMemcpyAsync(&s->d_reqs[r->slot], &R, sizeof(ServeReqDev), cudaMemcpyHostToDevice, s->s_h2d);
    if (e != cudaSuccess) return cuda_fail(e, "server: request copy");
    for (int js : new_jobs) {
        const unsigned long long pos = s->ring_tail++;
        const int ri = (int)(pos % (unsigned long long)s->ring_cap);
        s->h_ring[ri] = ((unsigned long long)(uint32_t)(pos + 1) << 32) | (uint32_t)js;
        e = cudaMemcpyAsync(&s->d_ring[ri], &s->h_ring[ri], sizeof(unsigned long long), cudaMemcpyHostToDevice,
                            s->s_h2d);
        if (e != cudaSuccess) return cuda_fail(e, "server: ring copy");
    }
    r->state = R_RUNNING;
    return KSIM_OK;
}

void ensure_loop(ksim_server *s)
{
    if (s->loop_running) {
        const cudaError_t q = cudaEventQuery(s->loop_done);
        if (q == cudaErrorNotReady) return;
        s->loop_running = false;
        if (q != cudaSuccess) {
            s->fatal = std::string("server loop kernel: ") + cudaGetErrorString(q);
            return;
        }
    }
    bool need = false;
    for (ServeRequest *r : s->running)
        if (r->loop && r->state == R_RUNNING) need = true;
    if (!need) return;
    // start after everything published so far has landed, with the exit word clear
    cudaError_t e = cudaEventRecord(s->h2d_mark, s->s_h2d);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s->s_loop, s->h2d_mark, 0);
    if (e == cudaSuccess) e = cudaMemsetAsync(&s->d_ctl->exiting, 0, sizeof(int32_t), s->s_loop);
    if (e == cudaSuccess) {
        k_serve<<<s->grid, s->lcfg.threads, s->smem, s->s_loop>>>(s->d_jobs, s->d_reqs, s->d_ring, s->ring_cap,
                                                                   s->d_ctl, s->d_done,
                                                                   (long long)s->cfg.idle_us * 1000ll);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(s->loop_done, s->s_loop);
    if (e != cudaSuccess) {
        s->fatal = std::string("server loop launch: ") + cudaGetErrorString(e);
        return;
    }
    s->loop_running = true;
    s->st.loop_launches += 1;
}

// One pass of the scheduler (caller holds mu).  Returns true if anything moved.
bool step(ksim_server *s)
{
    bool moved = false;
    // 1. admission, strictly in arrival order
    while (!s->pending.empty() && s->fatal.empty()) {
        ServeRequest *r = s->pending.front();
        AdmitNeed need = {Arena::round_up(std::max<int64_t>(r->f_bytes, 1), 256) + std::max<int64_t>(r->out_bytes, 1),
                          r->loop ? r->n_jobs : 0, r->loop ? r->n_jobs : 0};
        AdmitState state = {&s->arena, &s->req_slots, &s->job_slots, (int64_t)s->ring_cap, s->jobs_in_flight};
        const int a = admissible(need, state);
        if (a == 0) break;
        s->pending.pop_front();
        moved = true;
        if (a < 0) {
            finish(s, r, KSIM_ERR_OUT_OF_MEMORY, "request exceeds the server's arena / job table");
            s->cv_done.notify_all();
            continue;
        }
        const ksim_status st = admit(s, r);
        if (st != KSIM_OK) {
            const std::string err = ksim_last_error();
            release(s, r);
            finish(s, r, st, err);
            s->cv_done.notify_all();
            if (st == KSIM_ERR_CUDA) s->fatal = err;
            continue;
        }
        s->running.push_back(r);
    }
    // 2. keep the loop alive while loop work is in flight
    if (s->fatal.empty()) ensure_loop(s);
    // 3. completions
    for (size_t i = 0; i < s->running.size();) {
        ServeRequest *r = s->running[i];
        bool done = false;
        if (r->state == R_RUNNING) {
            bool finished;
            if (r->loop) {
                finished = *(volatile uint32_t *)&s->h_done[r->slot] == r->seq;
            } else {
                const cudaError_t q = cudaEventQuery(r->ev);
                finished = q != cudaErrorNotReady;
                if (finished && q != cudaSuccess) s->fatal = std::string("side launch: ") + cudaGetErrorString(q);
            }
            if (finished) {
                moved = true;
                cudaError_t e = cudaSuccess;
                if (!r->loop) e = cudaStreamWaitEvent(s->s_d2h, r->ev, 0);
                if (r->ev) {
                    cudaEventDestroy(r->ev);
                    r->ev = nullptr;
                }
                const int64_t f_region = Arena::round_up(std::max<int64_t>(r->f_bytes, 1), 256);
                if (e == cudaSuccess && r->out_bytes > 0)
                    e = cudaMemcpyAsync(r->out, s->d_arena + r->arena_off + f_region, (size_t)r->out_bytes,
                                        cudaMemcpyDeviceToHost, s->s_d2h);
                if (e == cudaSuccess && r->loop)
                    e = cudaMemcpyAsync(&s->h_reqs_back[r->slot], &s->d_reqs[r->slot], sizeof(ServeReqDev),
                                        cudaMemcpyDeviceToHost, s->s_d2h);
                if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->ev, cudaEventDisableTiming);
                if (e == cudaSuccess) e = cudaEventRecord(r->ev, s->s_d2h);
                if (e != cudaSuccess) {
                    s->fatal = std::string("server output copy: ") + cudaGetErrorString(e);
                } else {
                    r->state = R_COPYING;
                }
            }
        }
        if (r->state == R_COPYING) {
            const cudaError_t q = cudaEventQuery(r->ev);
            if (q != cudaErrorNotReady) {
                moved = true;
                ksim_status st = KSIM_OK;
                std::string err;
                if (q != cudaSuccess) {
                    st = KSIM_ERR_CUDA;
                    err = std::string("server output copy: ") + cudaGetErrorString(q);
                } else if (r->loop && (s->h_reqs_back[r->slot].flags & KSIM_FLAG_WAIT_TIMEOUT)) {
                    st = KSIM_ERR_TIMEOUT;
                    err = "a staging wait of the serving loop timed out";
                }
                release(s, r);
                finish(s, r, st, err);
                done = true;
            }
        }
        if (done) {
            s->running.erase(s->running.begin() + (long)i);
            s->cv_done.notify_all();
        } else {
            ++i;
        }
    }
    // 4. a CUDA failure fails everything still queued or running
    if (!s->fatal.empty()) {
        for (ServeRequest *r : s->running) {
            release(s, r);
            finish(s, r, KSIM_ERR_CUDA, s->fatal);
        }
        s->running.clear();
        for (ServeRequest *r : s->pending) finish(s, r, KSIM_ERR_CUDA, s->fatal);
        s->pending.clear();
        s->cv_done.notify_all();
    }
    return moved;
}

void worker_main(ksim_server *s)
{
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        const bool moved = step(s);
        const bool busy = !s->running.empty() || !s->pending.empty();
        if (s->stopping && s->running.empty() && s->pending.empty()) break;
        if (moved) continue;
        if (busy) {
            // device work in flight: poll again soon
            s->cv_work.wait_for(lk, std::chrono::microseconds(20));
        } else {
            s->cv_work.wait_for(lk, std::chrono::milliseconds(5));
        }
    }
}

}  // namespace
}  // namespace ksim

extern "C" {

ksim_status ksim_server_create(const ksim_server_config *cfg_in, ksim_server **out)
{
    if (!out) return fail(KSIM_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (ksim_device_count() <= 0) return fail(KSIM_ERR_NO_DEVICE, "no CUDA device is visible");
    ksim_server_config cfg = {};
    if (cfg_in) cfg = *cfg_in;
    if (cfg.device < 0 && cudaGetDevice(&cfg.device) != cudaSuccess)
        return fail(KSIM_ERR_NO_DEVICE, "cudaGetDevice failed");
    if (cfg.arena_bytes <= 0) cfg.arena_bytes = (int64_t)1 << 30;
    if (cfg.max_requests <= 0) cfg.max_requests = 1024;
    if (cfg.max_jobs <= 0) cfg.max_jobs = 4096;
    if (cfg.threads <= 0) cfg.threads = 128;
    if (cfg.slot_bytes <= 0) cfg.slot_bytes = 16384;
    if (cfg.idle_us <= 0) cfg.idle_us = 2000;
    if (cfg.threads > 256 || (cfg.threads & 31))
        return fail(KSIM_ERR_INVALID_ARGUMENT, "threads must be a multiple of 32 in [32, 256]");
    if ((cfg.slot_bytes & 15) || sample_smem_bytes(cfg.slot_bytes, true, 4, cfg.threads) > 227 * 1024)
        return fail(KSIM_ERR_INVALID_ARGUMENT,
                    "slot_bytes must be a multiple of 16, and two slots with the parity scratch fit in 227 KiB");
    std::unique_ptr<ksim_server> s(new ksim_server());
    s->device = cfg.device;
    s->cfg = cfg;
    s->lcfg.threads = cfg.threads;
    s->lcfg.staged = 1;
    s->lcfg.slot_bytes = cfg.slot_bytes;
    s->ring_cap = cfg.max_jobs;
    DeviceGuard g(cfg.device);
    if (!g.ok) return fail(KSIM_ERR_INVALID_ARGUMENT, "cannot select device " + std::to_string(cfg.device));

    auto bail = [&](cudaError_t e, const char *what) {
        ksim_server_destroy(s.release());
        return cuda_fail(e, what);
    };
    cudaError_t e = cudaMalloc(&s->d_arena, (size_t)cfg.arena_bytes);
    if (e != cudaSuccess) return bail(e, "server arena");
    s->arena.reset(cfg.arena_bytes, 256);
    s->req_slots.reset(cfg.max_requests);
    s->job_slots.reset(cfg.max_jobs);
    if ((e = cudaMalloc(&s->d_jobs, sizeof(ServeJob) * cfg.max_jobs)) != cudaSuccess) return bail(e, "job table");
    if ((e = cudaMallocHost(&s->h_jobs, sizeof(ServeJob) * cfg.max_jobs)) != cudaSuccess) return bail(e, "job table");
    if ((e = cudaMalloc(&s->d_reqs, sizeof(ServeReqDev) * cfg.max_requests)) != cudaSuccess)
        return bail(e, "request table");
    if ((e = cudaMallocHost(&s->h_reqs, sizeof(ServeReqDev) * cfg.max_requests)) != cudaSuccess)
        return bail(e, "request table");
    if ((e = cudaMallocHost(&s->h_reqs_back, sizeof(ServeReqDev) * cfg.max_requests)) != cudaSuccess)
        return bail(e, "request table");
    if ((e = cudaMalloc(&s->d_ring, sizeof(unsigned long long) * s->ring_cap)) != cudaSuccess)
        return bail(e, "job ring");
    if ((e = cudaMemset(s->d_ring, 0, sizeof(unsigned long long) * s->ring_cap)) != cudaSuccess)
        return bail(e, "job ring");
    if ((e = cudaMallocHost(&s->h_ring, sizeof(unsigned long long) * s->ring_cap)) != cudaSuccess)
        return bail(e, "job ring");
    if ((e = cudaMalloc(&s->d_ctl, sizeof(ServeCtl))) != cudaSuccess) return bail(e, "loop control");
    if ((e = cudaMemset(s->d_ctl, 0, sizeof(ServeCtl))) != cudaSuccess) return bail(e, "loop control");
    if ((e = cudaHostAlloc(&s->h_done, sizeof(uint32_t) * cfg.max_requests, cudaHostAllocMapped)) != cudaSuccess)
        return bail(e, "completion flags");
    std::fill(s->h_done, s->h_done + cfg.max_requests, 0u);
    if ((e = cudaHostGetDevicePointer((void **)&s->d_done, s->h_done, 0)) != cudaSuccess)
        return bail(e, "completion flags");
    if ((e = cudaMallocHost(&s->h_stop, sizeof(int32_t))) != cudaSuccess) return bail(e, "stop word");
    *s->h_stop = 1;
    for (cudaStream_t *st : {&s->s_h2d, &s->s_d2h, &s->s_loop, &s->s_side})
        if ((e = cudaStreamCreateWithFlags(st, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "streams");
    if ((e = cudaEventCreateWithFlags(&s->loop_done, cudaEventDisableTiming)) != cudaSuccess) return bail(e, "events");
    if ((e = cudaEventCreateWithFlags(&s->h2d_mark, cudaEventDisableTiming)) != cudaSuccess) return bail(e, "events");
    s->smem = sample_smem_bytes(cfg.slot_bytes, true, 4, cfg.threads);
    if ((e = cudaFuncSetAttribute(k_serve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s->smem)) != cudaSuccess)
        return bail(e, "loop kernel attributes");
    int active = 0, sms = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&active, k_serve, cfg.threads, s->smem)) != cudaSuccess)
        return bail(e, "loop kernel occupancy");
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, cfg.device);
    const int per_sm = cfg.ctas_per_sm > 0 ? std::min(cfg.ctas_per_sm, std::max(active, 1)) : std::max(active, 1);
    s->grid = std::max(1, per_sm * sms);
    s->st.arena_capacity = cfg.arena_bytes;
    ksim_server *raw = s.release();
    raw->worker = std::thread(worker_main, raw);
    *out = raw;
    return KSIM_OK;
}

ksim_status ksim_server_submit(ksim_server *s, ksim_program *p, const uint8_t *f, int64_t B, int64_t n_f_cols,
                               int64_t f_row_stride, uint64_t seed, int32_t rng_mode, uint8_t *out,
                               int64_t *request_id)
{
    if (!s || !p || !request_id) return fail(KSIM_ERR_INVALID_ARGUMENT, "server, program or request_id is NULL");
    if (p->device != s->device) return fail(KSIM_ERR_INVALID_ARGUMENT, "program lives on another device");
    if (B < 0 || n_f_cols < 0) return fail(KSIM_ERR_INVALID_ARGUMENT, "B and n_f_cols must be >= 0");
    if (rng_mode != KSIM_RNG_XORSHIFT && rng_mode != KSIM_RNG_PHILOX)
        return fail(KSIM_ERR_INVALID_ARGUMENT, "rng_mode must be KSIM_RNG_XORSHIFT or KSIM_RNG_PHILOX");
    if (n_f_cols < p->min_f_cols)
        return fail(KSIM_ERR_INVALID_ARGUMENT, "f has " + std::to_string(n_f_cols) + " columns; f_selection needs " +
                                                   std::to_string(p->min_f_cols));
    if (f_row_stride < n_f_cols) return fail(KSIM_ERR_INVALID_ARGUMENT, "f_row_stride < n_f_cols");
    if (B > 0 && ((n_f_cols > 0 && !f) || (p->n_outputs > 0 && !out)))
        return fail(KSIM_ERR_INVALID_ARGUMENT, "f or out is NULL");
    std::unique_ptr<ServeRequest> r(new ServeRequest());
    r->prog = p;
    r->f = f;
    r->out = out;
    r->B = B;
    r->n_f_cols = n_f_cols;
    r->f_stride = f_row_stride;
    r->f_bytes = B * n_f_cols;
    r->out_bytes = B * p->n_outputs;
    r->seed = seed;
    r->rng_mode = rng_mode;
    r->loop = words_of(p) <= 4;
    for (const ProgramPart &part : p->parts) r->n_jobs += part.comp->img.n_out > 0 ? 1 : 0;
    r->t_submit = Clock::now();
    // every component needs its chunk directory for the loop's slot size
    if (r->loop)
        for (const ProgramPart &part : p->parts) {
            if (part.comp->img.max_term_bytes > s->lcfg.slot_bytes)
                r->loop = false;  // a term larger than the loop's slot: plain launch
        }
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) return fail(KSIM_ERR_INVALID_ARGUMENT, "server is shutting down");
    if (!s->fatal.empty()) return fail(KSIM_ERR_CUDA, s->fatal);
    const int64_t footprint = Arena::round_up(std::max<int64_t>(r->f_bytes, 1), 256) + std::max<int64_t>(r->out_bytes, 1);
    if (!s->arena.ever_fits(footprint))
        return fail(KSIM_ERR_OUT_OF_MEMORY, "request needs " + std::to_string(footprint) +
                                                " arena bytes; the server has " + std::to_string(s->arena.capacity()));
    if (r->loop && r->n_jobs > s->job_slots.size())
        return fail(KSIM_ERR_UNSUPPORTED, "program has more components than the server's job table");
    r->id = s->next_id++;
    *request_id = r->id;
    ServeRequest *raw = r.get();
    s->all[r->id] = std::move(r);
    s->st.submitted += 1;
    if (raw->B == 0 || raw->prog->n_outputs == 0) {
        finish(s, raw, KSIM_OK, "");
        s->cv_done.notify_all();
        return KSIM_OK;
    }
    s->pending.push_back(raw);
    s->cv_work.notify_one();
    return KSIM_OK;
}

ksim_status ksim_server_poll(ksim_server *s, int64_t request_id, int32_t *done)
{
    if (!s || !done) return fail(KSIM_ERR_INVALID_ARGUMENT, "server or done is NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(request_id);
    if (it == s->all.end()) return fail(KSIM_ERR_NOT_FOUND, "unknown request id " + std::to_string(request_id));
    *done = it->second->state == R_DONE ? 1 : 0;
    return KSIM_OK;
}

ksim_status ksim_server_wait(ksim_server *s, int64_t request_id, int32_t timeout_ms, double *latency_s,
                             double *done_time_s)
{
    if (!s) return fail(KSIM_ERR_INVALID_ARGUMENT, "server is NULL");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(request_id);
    if (it == s->all.end()) return fail(KSIM_ERR_NOT_FOUND, "unknown request id " + std::to_string(request_id));
    ServeRequest *r = it->second.get();
    auto pred = [&] { return r->state == R_DONE; };
    if (timeout_ms < 0) {
        s->cv_done.wait(lk, pred);
    } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred)) {
        return fail(KSIM_ERR_TIMEOUT, "request " + std::to_string(request_id) + " is not done yet");
    }
    if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
    if (done_time_s) *done_time_s = to_seconds(r->t_done);
    const ksim_status st = r->status;
    const std::string err = r->error;
    s->all.erase(it);
    if (st != KSIM_OK) return fail(st, err);
    return KSIM_OK;
}

ksim_status ksim_server_cancel(ksim_server *s, int64_t request_id)
{
    if (!s) return fail(KSIM_ERR_INVALID_ARGUMENT, "server is NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(request_id);
    if (it == s->all.end()) return fail(KSIM_ERR_NOT_FOUND, "unknown request id " + std::to_string(request_id));
    ServeRequest *r = it->second.get();
    if (r->state != R_PENDING)
        return fail(KSIM_ERR_INVALID_ARGUMENT, "request " + std::to_string(request_id) + " is already admitted");
    s->pending.erase(std::find(s->pending.begin(), s->pending.end(), r));
    finish(s, r, KSIM_ERR_CANCELLED, "cancelled before admission");
    s->cv_done.notify_all();
    return KSIM_OK;
}

ksim_status ksim_server_get_stats(ksim_server *s, ksim_server_stats *out)
{
    if (!s || !out) return fail(KSIM_ERR_INVALID_ARGUMENT, "server or out is NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->st;
    out->pending = (int64_t)s->pending.size();
    out->in_flight = (int64_t)s->running.size();
    out->arena_in_use = s->arena.in_use();
    out->arena_capacity = s->arena.capacity();
    return KSIM_OK;
}

void ksim_server_destroy(ksim_server *s)
{
    if (!s) return;
    DeviceGuard g(s->device);
    if (s->worker.joinable()) {
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->stopping = true;
            for (ServeRequest *r : s->pending) finish(s, r, KSIM_ERR_CANCELLED, "server destroyed");
            s->pending.clear();
            s->cv_done.notify_all();
            s->cv_work.notify_all();
        }
        s->worker.join();
    }
    if (s->d_ctl && s->h_stop && s->s_h2d) {
        // tell a loop that is still idling to leave now
        cudaMemcpyAsync(&s->d_ctl->stop, s->h_stop, sizeof(int32_t), cudaMemcpyHostToDevice, s->s_h2d);
        cudaStreamSynchronize(s->s_h2d);
    }
    for (cudaStream_t st : {s->s_loop, s->s_side, s->s_h2d, s->s_d2h})
        if (st) cudaStreamSynchronize(st);
    for (cudaStream_t st : {s->s_loop, s->s_side, s->s_h2d, s->s_d2h})
        if (st) cudaStreamDestroy(st);
    if (s->loop_done) cudaEventDestroy(s->loop_done);
    if (s->h2d_mark) cudaEventDestroy(s->h2d_mark);
    for (auto &kv : s->all)
        if (kv.second->ev) cudaEventDestroy(kv.second->ev);
    if (s->d_arena) cudaFree(s->d_arena);
    if (s->d_jobs) cudaFree(s->d_jobs);
    if (s->h_jobs) cudaFreeHost(s->h_jobs);
    if (s->d_reqs) cudaFree(s->d_reqs);
    if (s->h_reqs) cudaFreeHost(s->h_reqs);
    if (s->h_reqs_back) cudaFreeHost(s->h_reqs_back);
    if (s->d_ring) cudaFree(s->d_ring);
    if (s->h_ring) cudaFreeHost(s->h_ring);
    if (s->d_ctl) cudaFree(s->d_ctl);
    if (s->h_done) cudaFreeHost(s->h_done);
    if (s->h_stop) cudaFreeHost(s->h_stop);
    delete s;
}

}  // extern "C"
