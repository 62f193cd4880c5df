/*
 * ksim_b200.h — C ABI of the B200-native ksim sampler.
 *
 * This is the drop-in boundary for ksim's sampling hot path
 * (FlatProgram -> samples).  Every entry point takes plain pointers and sizes;
 * no C++, Python or torch type crosses it.  Device work runs in hand-written
 * sm_100a CUDA kernels inside libksim_b200.so.
 *
 * Reference interfaces replaced (paths inside the ksim project):
 *   kokkos_sim.Component(graphs, num_f)        src/cpp/ksim/kokkos_sim.cpp:67-152
 *   Component.sample(f_sel, seed)              src/cpp/ksim/kokkos_sim.cpp:188-241
 *   Component.eval_abs(graph, params)          src/cpp/ksim/kokkos_sim.cpp:157-185
 *   Component.n_out                            src/cpp/ksim/kokkos_sim.cpp:250-251
 *   KokkosProgramSampler.sample(f, seed)       src/python/ksim/sample/sampler.py:57-67
 *   per-graph dict layout (_graph_to_dict)     src/python/ksim/sample/sampler.py:21-43
 *
 * Errors are status codes; the message of the last failing call on the
 * calling thread is available from ksim_last_error().  KSIM_ERR_INVALID_ARGUMENT
 * is what the reference reports as std::invalid_argument (Python ValueError).
 */
#ifndef KSIM_B200_H
#define KSIM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KSIM_B200_ABI_VERSION 1

typedef enum ksim_status {
    KSIM_OK = 0,
    KSIM_ERR_INVALID_ARGUMENT = 1, /* bad shape / count / pointer (ValueError) */
    KSIM_ERR_MALFORMED_PROGRAM = 2, /* a graph's arrays are inconsistent        */
    KSIM_ERR_CUDA = 3,              /* a CUDA runtime call failed               */
    KSIM_ERR_OUT_OF_MEMORY = 4,     /* device or pinned host allocation failed  */
    KSIM_ERR_TIMEOUT = 5,           /* a bounded device wait ran out            */
    KSIM_ERR_UNSUPPORTED = 6,       /* size beyond what this build handles      */
    KSIM_ERR_NOT_FOUND = 7,         /* unknown request / handle                 */
    KSIM_ERR_CANCELLED = 8,         /* request cancelled before completion      */
    KSIM_ERR_NO_DEVICE = 9,         /* no CUDA device visible                   */
    KSIM_ERR_INTERNAL = 10
} ksim_status;

/* Uniform streams for the per-output Bernoulli draw.
 *   KSIM_RNG_XORSHIFT: the reference's per-shot stream, bit-identical to
 *     kokkos_sim for the same seed (seed mixing kokkos_sim.cpp:215-217,
 *     xorshift64 13/7/17 kokkos_sim.cpp:43-46).
 *   KSIM_RNG_PHILOX: counter-based Philox4x32-10 (Salmon et al., SC'11),
 *     key = (seed lo32, seed hi32), counter = (shot lo32, shot hi32, output, 0),
 *     u = ((x1:x0) >> 11) * 2^-53.  Any shot range can be recomputed alone. */
enum { KSIM_RNG_XORSHIFT = 0, KSIM_RNG_PHILOX = 1 };

/* Advisory status bits raised by the kernels (results are never changed). */
enum {
    KSIM_FLAG_INT64_RISK = 1u,      /* a Z[w] coefficient exceeded 2^62 before a multiply */
    KSIM_FLAG_PREV_NONPOSITIVE = 2u,/* a marginal |A| was <= 0 at a Bernoulli step       */
    KSIM_FLAG_NAN = 4u,             /* p1/prev was NaN                                   */
    KSIM_FLAG_WAIT_TIMEOUT = 8u     /* a bounded device wait gave up                     */
};

/* One FlatScalarGraph, exactly the 19 arrays of the reference's per-graph dict
 * (sampler.py:21-43), C-contiguous, borrowed for the duration of the call.
 * G = pf_phase_idx.shape[0], P = np_params.shape[2], T* = family widths
 * (kokkos_sim.cpp:98-103).  Arrays of a zero-sized shape may be NULL. */
typedef struct ksim_graph_desc {
    int32_t G, P, Tnp, Thp, Tpp, Tph;
    const uint8_t *np_phases;   /* (G,Tnp)   */
    const uint8_t *np_params;   /* (G,Tnp,P) */
    const int32_t *np_counts;   /* (G,)      */
    const uint8_t *hp_coeffs;   /* (G,Thp)   */
    const uint8_t *hp_params;   /* (G,Thp,P) */
    const uint8_t *pp_psi_c;    /* (G,Tpp)   */
    const uint8_t *pp_psi_p;    /* (G,Tpp,P) */
    const uint8_t *pp_phi_c;    /* (G,Tpp)   */
    const uint8_t *pp_phi_p;    /* (G,Tpp,P) */
    const uint8_t *ph_alpha;    /* (G,Tph)   */
    const uint8_t *ph_alpha_p;  /* (G,Tph,P) */
    const uint8_t *ph_beta;     /* (G,Tph)   */
    const uint8_t *ph_beta_p;   /* (G,Tph,P) */
    const int32_t *ph_counts;   /* (G,)      */
    const uint8_t *pf_phase_idx;   /* (G,)   */
    const int32_t *pf_floatfactor; /* (G,4)  */
    const int32_t *pf_power2;      /* (G,)   */
    const float *pf_approx_f32;    /* (G,2) complex64 as float pairs */
    int32_t pf_has_approx;
} ksim_graph_desc;

typedef struct ksim_component ksim_component;
typedef struct ksim_program ksim_program;

/* ---- library ---------------------------------------------------------- */

/* Message of the last failing call on this thread ("" if none). */
const char *ksim_last_error(void);
int32_t ksim_abi_version(void);
/* Number of visible CUDA devices (0 when none; never fails). */
int32_t ksim_device_count(void);

/* ---- component: kokkos_sim.Component ----------------------------------- */

/* Validate, pack into the device structure-of-arrays image and upload.
 * Replaces KokkosTsimComponent(graphs, F), kokkos_sim.cpp:67-152.
 * device < 0 selects the calling thread's current device. */
ksim_status ksim_component_create(const ksim_graph_desc *graphs, int32_t n_graphs,
                                  int32_t num_f, int32_t device,
                                  ksim_component **out);
void ksim_component_destroy(ksim_component *c);
int32_t ksim_component_n_out(const ksim_component *c);   /* n_graphs - 1 */
int32_t ksim_component_num_f(const ksim_component *c);
int32_t ksim_component_n_graphs(const ksim_component *c);
int32_t ksim_component_words(const ksim_component *c);   /* 64-bit words per parameter vector */
int64_t ksim_component_image_bytes(const ksim_component *c);

/* Host buffers, synchronous.  f_sel: (B, num_f) uint8 C-contiguous; out:
 * (B, max(n_out,1)) uint8.  Replaces Component.sample, kokkos_sim.cpp:188-241
 * (bit-identical to it with rng_mode = KSIM_RNG_XORSHIFT).  Runs as the
 * pipelined host call of ksim_program_sample on the component alone (built
 * on the first call, freed with the component), so copies overlap sampling;
 * page-locked buffers overlap best. */
ksim_status ksim_component_sample(ksim_component *c, const uint8_t *f_sel, int64_t B,
                                  uint64_t seed, int32_t rng_mode, uint8_t *out);

/* Device buffers, asynchronous on `stream` (a cudaStream_t; NULL = legacy
 * default stream).  Shot s of this call uses shot index shot_offset + s for
 * its uniforms, so a shot range split across calls or GPUs reproduces the
 * single-call result.  out_stride = bytes between output rows (>= n_out);
 * out_col0 = first column written.  amp (nullable): (B, n_out+1) float64 of
 * |A_k| per graph, for parity checks. */
ksim_status ksim_component_sample_device(ksim_component *c, const uint8_t *d_f_sel,
                                         int64_t B, int64_t shot_offset, uint64_t seed,
                                         int32_t rng_mode, uint8_t *d_out,
                                         int64_t out_stride, int64_t out_col0,
                                         double *d_amp, void *stream);

/* The same sampling as ksim_component_sample_device (same arguments, same
 * bits, same |A_k|), for callers that cannot allocate device memory: code
 * whose HBM belongs to another allocator or is reserved up front, or that must
 * not take the device-wide synchronisation a cudaMalloc / cudaFree may cause
 * in a latency-critical loop.  No reference counterpart: kokkos_sim always
 * allocates its Views inside Component.sample.
 *
 * The call allocates nothing.  Its scratch (the staging chunk directory) is
 * one fixed array of KSIM_NOALLOC_SCRATCH_BYTES in device memory, loaded with
 * the library on every GPU that uses it and held until the process exits.  A
 * component needing more than KSIM_NOALLOC_MAX_CHUNKS staging chunks (or an
 * image above 4 GiB) is rejected with KSIM_ERR_UNSUPPORTED.  The directory
 * reaches the array as the by-value parameter of a one-CTA kernel queued on
 * `stream` before the sampling kernel, so no host buffer is copied and the
 * call does not wait for the stream.  The kernels' KSIM_FLAG_* bits (wait
 * timeout, int64 risk, ...) go to the component's status word, read with
 * ksim_component_status as for every other sampling call.  The first call on
 * a device looks up the array's device address; make that first call before
 * any stream capture.  Every call shares the array and leaves its directory
 * behind, so calls that overlap on the GPU (other streams, other threads)
 * race on it: issue them on one stream. */
#define KSIM_NOALLOC_SCRATCH_BYTES 32768
#define KSIM_NOALLOC_MAX_CHUNKS 1024
ksim_status ksim_component_sample_device_noalloc(ksim_component *c, const uint8_t *d_f_sel,
                                                 int64_t B, int64_t shot_offset, uint64_t seed,
                                                 int32_t rng_mode, uint8_t *d_out,
                                                 int64_t out_stride, int64_t out_col0,
                                                 double *d_amp, void *stream);

/* |amplitude| of graph `graph` for B explicit parameter rows (B, P) uint8.
 * Replaces Component.eval_abs, kokkos_sim.cpp:157-185.  Host buffers. */
ksim_status ksim_component_eval_abs(ksim_component *c, int32_t graph, const uint8_t *params,
                                    int64_t B, int64_t P, double *out);
/* Complex amplitude (B, 2) float64 (re, im) of the same evaluation. */
ksim_status ksim_component_eval(ksim_component *c, int32_t graph, const uint8_t *params,
                                int64_t B, int64_t P, double *out_re_im);
/* Per-term exact Z[w] numerators: out (B, G, 5) int64 = (a, b, c, d, pw) in
 * the basis (1, w, i, conj w) after the term's last renormalisation step
 * (zx_eval.hpp:101-165 schedule), before the prefactor power2. */
ksim_status ksim_component_eval_terms(ksim_component *c, int32_t graph, const uint8_t *params,
                                      int64_t B, int64_t P, int64_t *out);

/* OR of KSIM_FLAG_* raised by this component's kernels since the last reset. */
ksim_status ksim_component_status(ksim_component *c, uint32_t *flags, int32_t reset);

/* Launch shape of the plain sampler for this component: threads per CTA
 * (a multiple of 32, <= 256), whether term chunks are staged in shared memory
 * by TMA bulk copies, and the staging slot size in bytes (>= the largest term
 * record, a multiple of 16).  Zero / negative values keep the current value. */
ksim_status ksim_component_set_launch(ksim_component *c, int32_t threads, int32_t staged,
                                      int32_t slot_bytes);
ksim_status ksim_component_get_launch(const ksim_component *c, int32_t *threads, int32_t *staged,
                                      int32_t *slot_bytes);
/* Bound of the staging waits of this component's sampling kernels (plain,
 * batched, served and allocation-free), in non-blocking polls of the
 * mbarrier 64 ns apart: a wait that runs out raises KSIM_FLAG_WAIT_TIMEOUT,
 * the CTA waits (with the built-in bound) for the copies it issued and leaves
 * without writing its shots, and the synchronous host calls report
 * KSIM_ERR_TIMEOUT (and clear the flag they report).  0 restores the built-in
 * bound (2^22 blocking try_wait polls).  Batches and server jobs take the
 * value in force when they are created or admitted.  The reference has no bounded waits
 * (kokkos_sim.cpp:188-241 fences without a limit); this is the failure
 * detector's knob, and a small value lets a test see it fire. */
ksim_status ksim_component_set_wait_limit(ksim_component *c, int64_t polls);
/* Image statistics: terms, terms on the exact (overflow-risk) path, columns,
 * largest term record in bytes. */
ksim_status ksim_component_stats(const ksim_component *c, int64_t *n_terms, int64_t *n_slow_terms,
                                 int64_t *n_columns, int64_t *max_term_bytes);

/* ---- program: KokkosProgramSampler ------------------------------------- */

/* A FlatProgram: components (borrowed, must outlive the program, all on one
 * device), each with its f_selection (columns of the full f matrix), and
 * output_order (distinct values, one per output of the concatenated
 * components).  Replaces KokkosProgramSampler.__init__, sampler.py:48-55. */
ksim_status ksim_program_create(ksim_component *const *comps, int32_t n_comps,
                                const int32_t *const *f_selection, const int32_t *f_sel_len,
                                const int32_t *output_order, int32_t n_outputs,
                                ksim_program **out);
void ksim_program_destroy(ksim_program *p);
int32_t ksim_program_n_outputs(const ksim_program *p);
/* Smallest row width an f matrix must have (max f_selection + 1). */
int32_t ksim_program_min_f_cols(const ksim_program *p);

/* f_params: (B, n_f_cols) uint8 host; out: (B, n_outputs) uint8 host.
 * Component k is seeded with seed + 0x9E37*k and the outputs are permuted by
 * argsort(output_order), as sampler.py:57-67 does; the f_selection gather and
 * the permutation run on the device.  Large calls are split into chunks of
 * shots whose copies overlap the sampling of their neighbours (page-locked
 * host buffers let the copies run asynchronously). */
ksim_status ksim_program_sample(ksim_program *p, const uint8_t *f_params, int64_t B,
                                int64_t n_f_cols, uint64_t seed, int32_t rng_mode, uint8_t *out);
/* Bit-packed host I/O (no reference counterpart; it cuts the PCIe bytes of
 * ksim_program_sample 8x): f_packed has B rows of ceil(n_f_cols/8) bytes and
 * out_packed B rows of ceil(n_outputs/8) bytes; column c of a row is bit c%8
 * of byte c/8 (numpy.packbits(..., bitorder="little")).  The bits are those of
 * ksim_program_sample. */
ksim_status ksim_program_sample_packed(ksim_program *p, const uint8_t *f_packed, int64_t B,
                                       int64_t n_f_cols, uint64_t seed, int32_t rng_mode,
                                       uint8_t *out_packed);
/* Same on device buffers, asynchronous on `stream`. */
ksim_status ksim_program_sample_device(ksim_program *p, const uint8_t *d_f_params, int64_t B,
                                       int64_t n_f_cols, int64_t shot_offset, uint64_t seed,
                                       int32_t rng_mode, uint8_t *d_out, void *stream);

/* ---- noise: the f parameters drawn on the device ------------------------ */

/* A noise model: ChannelSampler(channel_probs, error_transform)
 * (src/python/ksim/compile/channels.py:531-576).  Channel i has n_bits[i]
 * error bits and 2^n_bits[i] outcome probabilities, concatenated in `probs`
 * (outcome index bit b = error bit b, channels.py:12-24); error_transform is
 * (num_f, num_e) uint8 row-major, num_e = sum of n_bits.  At creation,
 * channels that never fire are dropped and channels over identical
 * error-bit patterns are merged by XOR convolution (channels.py:398-429); the
 * rest are ordered by firing probability into runs of equal p, each with
 * integer skip thresholds floor((1 - p)^k 2^32).  The draw
 * (ChannelSampler.sample, channels.py:624-658) runs one thread per shot with
 * one counter-based Philox4x32-10 stream keyed by (seed, shot): within a run
 * the next firing channel is j + 1 + #{k : u < T_k} for a fresh draw u, the
 * outcome is the first whose conditional-CDF threshold exceeds the next draw,
 * and its f pattern is XORed in; the work per shot follows the channels that
 * fire. */
typedef struct ksim_noise ksim_noise;
ksim_status ksim_noise_create(const double *probs, const int32_t *n_bits, int32_t n_channels,
                              const uint8_t *error_transform, int32_t num_f, int32_t num_e,
                              int32_t device, ksim_noise **out);
void ksim_noise_destroy(ksim_noise *n);
int32_t ksim_noise_num_f(const ksim_noise *n);
int32_t ksim_noise_num_channels(const ksim_noise *n);   /* channels that can fire, after merging */
/* f rows (B x num_f bytes, f_stride apart) for shots shot_offset.. on the device. */
ksim_status ksim_noise_sample_device(ksim_noise *n, int64_t B, int64_t shot_offset, uint64_t seed,
                                     uint8_t *d_f, int64_t f_stride, void *stream);
/* The same into host memory (B x num_f bytes), synchronous. */
ksim_status ksim_noise_sample(ksim_noise *n, int64_t B, int64_t shot_offset, uint64_t seed,
                              uint8_t *f_host);
/* Draw f on the device and sample program p from it: only the outputs
 * (B x n_outputs bytes, host) cross PCIe.  Equals
 * ksim_program_sample(p, f, ...) with f = ksim_noise_sample(n, B, 0, noise_seed). */
ksim_status ksim_program_sample_noisy(ksim_program *p, ksim_noise *n, int64_t B, uint64_t noise_seed,
                                      uint64_t seed, int32_t rng_mode, uint8_t *out);

/* ---- batch: many programs in one persistent, graph-captured launch ------- */

/* One sampling job of a batch: a component over device rows of f bytes,
 * writing its outputs into device rows.  d_f_sel (nullable): component
 * parameter j reads row[d_f_sel[j]]; d_out_cols (nullable): output i goes to
 * column d_out_cols[i], else to out_col0 + i.  Shot s uses stream index
 * shot_offset + s, so a job's bits do not depend on what else is batched. */
typedef struct ksim_batch_job {
    ksim_component *comp;
    const uint8_t *d_f;
    int64_t f_stride;
    const int32_t *d_f_sel;
    uint8_t *d_out;
    int64_t out_stride, out_col0;
    const int32_t *d_out_cols;
    int64_t B, shot_offset;
    uint64_t seed;
    int32_t rng_mode;
} ksim_batch_job;

/* Launch shape of a batch (zero / negative fields take the defaults:
 * 128 threads, 14 KiB slots, CTAs per SM from occupancy, graph on).  The
 * shape applies to the jobs whose terms all run on 32-bit words with W <= 4
 * (the bulk of the work), drained by one persistent kernel; jobs with hybrid,
 * 64-bit or exact-path terms and jobs with W > 4 run in kernels of their own
 * (CTAs of 128; slots of at least 16 KiB for 64-bit, exact and W > 4 terms),
 * launched before it and overlapping it.  A work item is 2 x threads shots of a W <= 4 job
 * (two shots per thread) and threads shots of a wider one. */
typedef struct ksim_batch_tuning {
    int32_t threads;      /* threads per CTA (a multiple of 32, <= 256); see the item size above */
    int32_t slot_bytes;   /* staging slot, multiple of 16, >= the largest term of every 32-bit job */
    int32_t ctas_per_sm;  /* persistent CTAs per SM (<= occupancy limit) */
    int32_t use_graph;    /* 1: capture counter reset + kernels in a CUDA graph */
} ksim_batch_tuning;

typedef struct ksim_batch ksim_batch;

/* Components are borrowed and must outlive the batch; buffers are the
 * caller's.  No reference counterpart (the reference launches one component
 * at a time, sampler.py:60-64). */
ksim_status ksim_batch_create(const ksim_batch_job *jobs, int32_t n_jobs, const ksim_batch_tuning *tuning,
                              ksim_batch **out);
/* The batch job for component k of program p over device rows of the full f
 * matrix (f_stride bytes per row) and of the program's output matrix
 * (n_outputs bytes per row): f_selection gather, output permutation and the
 * per-component seed seed + 0x9E37*k as in KokkosProgramSampler.sample. */
ksim_status ksim_program_job(const ksim_program *p, int32_t k, const uint8_t *d_f, int64_t f_stride,
                             uint8_t *d_out, int64_t B, int64_t shot_offset, uint64_t seed, int32_t rng_mode,
                             ksim_batch_job *out);
int32_t ksim_program_n_components(const ksim_program *p);
/* Replace every job's seed (n_jobs values) before the next launch. */
ksim_status ksim_batch_set_seeds(ksim_batch *b, const uint64_t *seeds);
/* Enqueue the whole batch on `stream` (replays the captured graph). */
ksim_status ksim_batch_launch(ksim_batch *b, void *stream);
ksim_status ksim_batch_info(const ksim_batch *b, int64_t *n_items, int32_t *grid, int32_t *n_launches);
void ksim_batch_destroy(ksim_batch *b);

/* ---- serving: continuous batching with a device-resident request loop ---- */

/* No reference counterpart (kokkos_sim serves one synchronous call at a time,
 * kokkos_sim.cpp:188-241).  A server owns one device arena for request
 * buffers; a request is admitted, strictly in arrival order, once its HBM
 * footprint (f rows + output rows), a request slot, job-table slots and ring
 * room are free.  Admitted work is published to a device job ring that a
 * persistent kernel drains tile by tile: requests that arrive while others
 * run join the ring, and their tiles interleave with the running ones on the
 * device.  The loop kernel exits once no CTA has claimed work for idle_us and
 * is relaunched (full grid) by the server's scheduler thread when work arrives.  Results depend only on
 * (program, f, seed, rng_mode), never on what else is in flight.
 * Programs are borrowed: keep them alive until their requests finish. */
typedef struct ksim_server_config {
    int32_t device;          /* < 0: the calling thread's current device            */
    int64_t arena_bytes;     /* admission budget for request buffers (default 1 GiB) */
    int32_t max_requests;    /* request slots in flight (default 1024)               */
    int32_t max_jobs;        /* job-table slots in flight (default 4096)             */
    int32_t threads;         /* shots per tile = threads per CTA (default 128)       */
    int32_t slot_bytes;      /* staging slot of the loop kernel (default 16 KiB)     */
    int32_t ctas_per_sm;     /* loop CTAs per SM (default: occupancy limit)          */
    int32_t idle_us;         /* the loop exits after the whole grid claimed no work
                                for this long (default 2000)                         */
} ksim_server_config;

typedef struct ksim_server_stats {
    int64_t submitted, completed, failed, cancelled;
    int64_t shots_completed;
    int64_t loop_launches;   /* launches of the device-resident loop kernel */
    int64_t side_launches;   /* programs with > 256 parameter bits run as plain launches */
    int64_t pending, in_flight;
    int64_t arena_in_use, arena_capacity;
} ksim_server_stats;

typedef struct ksim_server ksim_server;

/* cfg may be NULL (all defaults); zero / negative fields take the defaults. */
ksim_status ksim_server_create(const ksim_server_config *cfg, ksim_server **out);
/* Queue a request: B shots of program p over host rows f (B rows of
 * n_f_cols bytes, f_row_stride bytes apart), seed and rng_mode as in
 * ksim_program_sample; results go to host `out` (B x n_outputs bytes) when
 * the request completes.  f and out must stay valid until then; page-locked
 * buffers let the copies overlap.  A request larger than the whole arena is
 * rejected with KSIM_ERR_OUT_OF_MEMORY. */
ksim_status ksim_server_submit(ksim_server *s, ksim_program *p, const uint8_t *f, int64_t B,
                               int64_t n_f_cols, int64_t f_row_stride, uint64_t seed,
                               int32_t rng_mode, uint8_t *out, int64_t *request_id);
/* Block until the request finishes (timeout_ms < 0: no limit; on expiry
 * KSIM_ERR_TIMEOUT and the request stays queued).  Returns the request's own
 * status (KSIM_ERR_CANCELLED, KSIM_ERR_TIMEOUT for a device wait that ran
 * out, ...).  latency_s (nullable): submit -> results in `out`, seconds;
 * done_time_s (nullable): completion time on the CLOCK_MONOTONIC clock.
 * A finished request is forgotten once waited on. */
ksim_status ksim_server_wait(ksim_server *s, int64_t request_id, int32_t timeout_ms,
                             double *latency_s, double *done_time_s);
/* done = 1 when finished (then ksim_server_wait returns at once). */
ksim_status ksim_server_poll(ksim_server *s, int64_t request_id, int32_t *done);
/* Cancel a request that has not been admitted yet (KSIM_ERR_NOT_FOUND for
 * an unknown id, KSIM_ERR_INVALID_ARGUMENT once it is on the device). */
ksim_status ksim_server_cancel(ksim_server *s, int64_t request_id);
ksim_status ksim_server_get_stats(ksim_server *s, ksim_server_stats *out);
/* Stop the loop, finish or cancel what is queued, free everything. */
void ksim_server_destroy(ksim_server *s);

/* ---- measurement --------------------------------------------------------- */

/* The roofline numerator: int32 operations one shot costs on a component in
 * the formulation the kernels run (32-bit words for terms proven below 2^31,
 * 64-bit words otherwise, the reference's step-by-step arithmetic for terms
 * on the exact path), and how many terms take each path (paths[0] 32-bit,
 * paths[1] 64-bit, paths[2] exact, paths[3] hybrid: NodePhases on 32-bit
 * words, the rest on 64-bit; nullable, 4 entries).  Host only: no device is
 * needed.  No reference counterpart. */
ksim_status ksim_work_model(const ksim_graph_desc *graphs, int32_t n_graphs, int32_t num_f,
                            double *ops_per_shot, int64_t *paths);

/* Integer-pipe throughput of this GPU for the sampler's instruction mix
 * (32-bit add / shift / logic), in int32 lane-operations per second: the
 * roofline denominator of the sampling kernels.  No reference counterpart. */
ksim_status ksim_measure_int_peak(int32_t device, double *ops_per_s, double *ms);
/* Integer ALU throughput alone (three-input add and three-input logic
 * chains, no shifts, multiplies or popcounts), in int32 lane-operations per
 * second: the ceiling of the pure add / logic part of the sampler's work.
 * No reference counterpart. */
ksim_status ksim_measure_alu_peak(int32_t device, double *ops_per_s, double *ms);

#ifdef __cplusplus
}
#endif

#endif /* KSIM_B200_H */
