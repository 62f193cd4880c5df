// hostemu.cpp — TEST INFRASTRUCTURE ONLY.
//
// Runs the device term evaluator (ksim_b200/csrc/zring.cuh) on the CPU over
// the packed image (ksim_b200/csrc/image.cpp), so the tests can check the
// packing, the valuation-scheduled renormalisation and the overflow-safety
// split against the oracle without a GPU.  It is never loaded by the
// package; tests/conftest.py builds it with g++.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "hostio.h"
#include "image.h"
#include "serve_sched.h"
#include "zring.cuh"

using namespace ksim;

namespace {
std::string g_err;

template <int W>
void pack_row(const uint8_t *row, int64_t n, uint64_t (&v)[W])
{
    for (int w = 0; w < W; ++w) v[w] = 0;
    for (int64_t c = 0; c < n && c < 64 * W; ++c) v[c >> 6] |= (uint64_t)(row[c] & 1u) << (c & 63);
    set_one_bit<W>(v);
}

// Modes 3 (per-term numerators) and 4 (complex amplitude): the same as 2 and
// 0, evaluated two rows at a time through the two-shots-per-thread path.
template <int W>
void eval_rows_pairs(const HostImage &img, int gi, const uint8_t *params, int64_t B, int64_t P, int mode,
                     void *out, uint32_t *risk_out)
{
    const GraphDir &gd = img.gdir[gi];
    uint32_t risk = 0;
    for (int64_t s = 0; s < B; s += 2) {
        const int n = B - s >= 2 ? 2 : 1;
        uint64_t v[2][W];
        pack_row<W>(params + s * P, P, v[0]);
        pack_row<W>(params + (s + n - 1) * P, P, v[1]);
        const uint8_t *p = img.bytes.data() + gd.stream_off;
        if (mode == 3) {
            for (int t = 0; t < gd.G; ++t) {
                const TermHdr h = load_hdr(p);
                TermOut r[2];
                p = eval_term_s<W, 2>(p, h, v, r);
                for (int k = 0; k < n; ++k) {
                    int64_t *o = (int64_t *)out + (s + k) * (int64_t)gd.G * 5 + 5 * t;
                    o[0] = (int64_t)r[k].z.a;
                    o[1] = (int64_t)r[k].z.b;
                    o[2] = (int64_t)r[k].z.c;
                    o[3] = (int64_t)r[k].z.d;
                    o[4] = r[k].pw;
                    risk |= r[k].risk;
                }
            }
        } else {
            double re[2] = {0, 0}, im[2] = {0, 0};
            eval_terms_s<W, 2>(p, (uint32_t)gd.G, v, re, im, risk, n == 2 ? 3u : 1u);
            for (int k = 0; k < n; ++k) {
                ((double *)out)[2 * (s + k)] = re[k];
                ((double *)out)[2 * (s + k) + 1] = im[k];
            }
        }
    }
    if (risk_out) *risk_out = risk;
}

template <int W>
void eval_rows(const HostImage &img, int gi, const uint8_t *params, int64_t B, int64_t P, int mode,
               void *out, uint32_t *risk_out)
{
    if (mode >= 3) return eval_rows_pairs<W>(img, gi, params, B, P, mode, out, risk_out);
    const GraphDir &gd = img.gdir[gi];
    uint32_t risk = 0;
    for (int64_t s = 0; s < B; ++s) {
        uint64_t v[W];
        pack_row<W>(params + s * P, P, v);
        const uint8_t *p = img.bytes.data() + gd.stream_off;
        if (mode == 2) {
            int64_t *o = (int64_t *)out + s * (int64_t)gd.G * 5;
            for (int t = 0; t < gd.G; ++t) {
                const TermHdr h = load_hdr(p);
                TermOut r;
                p = eval_term<W>(p, h, v, r);
                o[5 * t] = (int64_t)r.z.a;
                o[5 * t + 1] = (int64_t)r.z.b;
                o[5 * t + 2] = (int64_t)r.z.c;
                o[5 * t + 3] = (int64_t)r.z.d;
                o[5 * t + 4] = r.pw;
                risk |= r.risk;
            }
        } else {
            double re = 0, im = 0;
            eval_terms<W>(p, (uint32_t)gd.G, v, re, im, risk);
            ((double *)out)[2 * s] = re;
            ((double *)out)[2 * s + 1] = im;
        }
    }
    if (risk_out) *risk_out = risk;
}

template <int W>
void sample_rows(const HostImage &img, const uint8_t *f, int64_t B, uint64_t seed, int rng_mode, uint8_t *out,
                 double *amp)
{
    const int F = img.F, n_out = img.n_out, ncol = n_out > 1 ? n_out : 1;
    for (int64_t s = 0; s < B; ++s) {
        uint64_t v[W];
        pack_row<W>(f + s * F, F, v);
        uint64_t rng = xorshift_init(seed, (uint64_t)s);
        double prev = 0;
        for (int k = 0; k < img.n_graphs; ++k) {
            const int nm = k > 0 ? k - 1 : 0;
            uint64_t vk[W];
            for (int w = 0; w < W; ++w)
                vk[w] = (v[w] & bit_range(w, 0, F + nm)) | (k > 0 ? bit_range(w, F + nm, img.gdir[k].P) : 0);
            set_one_bit<W>(vk);
            double re = 0, im = 0;
            uint32_t risk = 0;
            eval_terms<W>(img.bytes.data() + img.gdir[k].stream_off, (uint32_t)img.gdir[k].G, vk, re, im, risk);
            const double mag = std::sqrt(re * re + im * im);
            if (amp) amp[s * (n_out + 1) + k] = mag;
            if (k == 0) {
                prev = mag;
                continue;
            }
            const int i = k - 1;
            const double u = rng_mode == 1 ? philox_uniform(seed, (uint64_t)s, (uint32_t)i) : xorshift_uniform(rng);
            const int bit = u < (mag / prev) ? 1 : 0;
            v[(F + i) >> 6] |= (uint64_t)bit << ((F + i) & 63);
            out[s * ncol + i] = (uint8_t)bit;
            prev = bit ? mag : prev - mag;
        }
    }
}

#define DISPATCH(W, CALL)                \
    switch (W) {                         \
    case 1: CALL(1); break;              \
    case 2: CALL(2); break;              \
    case 3: CALL(3); break;              \
    case 4: CALL(4); break;              \
    case 5: CALL(5); break;              \
    case 6: CALL(6); break;              \
    case 8: CALL(8); break;              \
    case 10: CALL(10); break;            \
    case 12: CALL(12); break;            \
    case 16: CALL(16); break;            \
    default: return 99;                  \
    }
}  // namespace

extern "C" {

const char *hostemu_error(void) { return g_err.c_str(); }

// stats: [W, n_terms, n_slow_terms, n_columns, max_term_bytes, n_narrow_terms, n_hybrid_terms]
int hostemu_stats(const ksim_graph_desc *g, int n, int F, int64_t *stats)
{
    HostImage img;
    int st = build_image(g, n, F, img, g_err);
    if (st) return st;
    stats[0] = img.W;
    stats[1] = img.n_terms;
    stats[2] = img.n_slow_terms;
    stats[3] = img.n_columns;
    stats[4] = img.max_term_bytes;
    stats[5] = img.n_narrow_terms;
    stats[6] = img.n_hybrid_terms;
    return 0;
}

int hostemu_eval(const ksim_graph_desc *g, int n, int F, int gi, const uint8_t *params, int64_t B, int64_t P,
                 int mode, void *out, uint32_t *risk)
{
    HostImage img;
    int st = build_image(g, n, F, img, g_err);
    if (st) return st;
#define CALL_EVAL(WW) eval_rows<WW>(img, gi, params, B, P, mode, out, risk)
    DISPATCH(img.W, CALL_EVAL)
    return 0;
}

int hostemu_sample(const ksim_graph_desc *g, int n, int F, const uint8_t *f, int64_t B, uint64_t seed,
                   int rng_mode, uint8_t *out, double *amp)
{
    HostImage img;
    int st = build_image(g, n, F, img, g_err);
    if (st) return st;
#define CALL_SAMPLE(WW) sample_rows<WW>(img, f, B, seed, rng_mode, out, amp)
    DISPATCH(img.W, CALL_SAMPLE)
    return 0;
}

uint32_t hostemu_valuation(const int64_t *z) { return zw_valuation(z); }

// The server's arena (serve_sched.h) driven by a script: ops[2i] = 0 allocates
// ops[2i+1] bytes (result: offset or -1), ops[2i] = 1 releases the offset
// returned by op number ops[2i+1] (result: 1 released, 0 refused).  state:
// in_use, largest_free, free_blocks, live_blocks after the script.
void hostemu_arena_run(int64_t capacity, int64_t align, const int64_t *ops, int n_ops, int64_t *results,
                       int64_t *state)
{
    Arena a(capacity, align);
    for (int i = 0; i < n_ops; ++i) {
        if (ops[2 * i] == 0) {
            results[i] = a.alloc(ops[2 * i + 1]);
        } else {
            const int64_t k = ops[2 * i + 1];
            results[i] = (k >= 0 && k < i) ? (a.release(results[k]) ? 1 : 0) : 0;
        }
    }
    state[0] = a.in_use();
    state[1] = a.largest_free();
    state[2] = a.free_blocks();
    state[3] = a.live_blocks();
}

// admissible() for an arena with one live block of `used` bytes at offset 0.
int hostemu_admissible(int64_t need_bytes, int need_jobs, int64_t need_ring, int64_t arena_cap, int64_t used,
                       int req_free, int req_total, int job_free, int job_total, int64_t ring_cap,
                       int64_t ring_in_flight)
{
    Arena a(arena_cap, 256);
    if (used > 0) a.alloc(used);
    SlotPool rq(req_total), jb(job_total);
    for (int i = req_free; i < req_total; ++i) rq.take();
    for (int i = job_free; i < job_total; ++i) jb.take();
    const AdmitNeed n = {need_bytes, need_jobs, need_ring};
    const AdmitState st = {&a, &rq, &jb, ring_cap, ring_in_flight};
    return admissible(n, st);
}

// The chunk plan of a host-buffer call (hostio.h): boundaries into out (at
// most cap), returns their count.
int hostemu_chunk_bounds(int64_t B, int64_t row_bytes, int64_t *out, int cap)
{
    const std::vector<int64_t> b = ksim::host_chunk_bounds(B, row_bytes);
    for (size_t i = 0; i < b.size() && (int)i < cap; ++i) out[i] = b[i];
    return (int)b.size();
}

int hostemu_copy_lag(const int64_t *bounds, int n, int64_t wave_shots, int max_lag)
{
    return ksim::host_copy_lag(std::vector<int64_t>(bounds, bounds + n), wave_shots, max_lag);
}

}  // extern "C"
