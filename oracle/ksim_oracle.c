/*
 * ksim_oracle.c — CPU restatement of ksim's sampling hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA kernels in
 * ksim_b200/csrc; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it.  The product never calls it.
 *
 * It restates, byte-per-bit and in the reference's operation order:
 *   - Z[w] arithmetic in the basis (1, w, i, conj w):   zx_eval.hpp:25-47
 *   - eval_graph (four term families + prefactor):      zx_eval.hpp:75-181
 *   - the per-shot autoregressive sample loop:          kokkos_sim.cpp:214-230
 *   - the per-shot xorshift stream and seed mixing:     kokkos_sim.cpp:43-46, 215-217
 * plus the counter-based Philox4x32-10 stream (Salmon et al., SC'11) that the
 * GPU path is also fed.  Parity of this restatement is pinned against the
 * reference's own zx_eval.hpp (built unmodified into oracle/_ref by
 * oracle/Makefile) and against the reference's numpy evaluate_flat through the
 * committed fixtures in tests/golden/.
 *
 * Build: oracle/Makefile (-O3 -ffp-contract=off -fwrapv, OpenMP over shots).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/ksim_b200.h"

typedef struct { int64_t a, b, c, d; } zw_t;

/* Product in the basis (1, w, i, conj w), from w*conj(w) = 1, w*w = i,
 * w*i = -conj(w), i*i = -1, i*conj(w) = w, conj(w)^2 = -i.  Unsigned
 * arithmetic gives the two's-complement wrap of the reference's int64. */
static inline zw_t zmul(zw_t x, zw_t y)
{
    uint64_t xa = (uint64_t)x.a, xb = (uint64_t)x.b, xc = (uint64_t)x.c, xd = (uint64_t)x.d;
    uint64_t ya = (uint64_t)y.a, yb = (uint64_t)y.b, yc = (uint64_t)y.c, yd = (uint64_t)y.d;
    zw_t r;
    r.a = (int64_t)(xa * ya + xb * yd - xc * yc + xd * yb);
    r.b = (int64_t)(xa * yb + xb * ya + xc * yd + xd * yc);
    r.c = (int64_t)(xa * yc + xb * yb + xc * ya - xd * yd);
    r.d = (int64_t)(xa * yd - xb * yc - xc * yb + xd * ya);
    return r;
}

/* One renormalisation step: halve when all four are even and not all zero. */
static inline void zreduce(zw_t *x, int64_t *pw)
{
    if ((x->a | x->b | x->c | x->d) != 0 &&
        ((x->a & 1) | (x->b & 1) | (x->c & 1) | (x->d & 1)) == 0) {
        x->a >>= 1; x->b >>= 1; x->c >>= 1; x->d >>= 1;
        *pw += 1;
    }
}

/* w^k for k in 0..7 in the same basis. */
static inline zw_t zunit(int k)
{
    static const int64_t t[8][4] = {
        {1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, -1},
        {-1, 0, 0, 0}, {0, -1, 0, 0}, {0, 0, -1, 0}, {0, 0, 0, 1}};
    zw_t r = {t[k][0], t[k][1], t[k][2], t[k][3]};
    return r;
}

/* Parameter bit j of one shot: j<F -> f byte, j<F+nm -> sampled m bit,
 * otherwise the "trying" bit (kokkos_sim.cpp:10-14, zx_eval.hpp:86-90). */
typedef struct {
    const uint8_t *f;   /* F bytes of this shot */
    const uint8_t *m;   /* sampled bits of this shot */
    int F, nm, trying;
} pvec_t;

static inline int pbit(const pvec_t *v, int j)
{
    if (j < v->F) return (int)v->f[j];
    if (j < v->F + v->nm) return (int)v->m[j - v->F];
    return v->trying;
}

static inline int parity_row(const uint8_t *row, int P, const pvec_t *v)
{
    int acc = 0;
    for (int j = 0; j < P; ++j) acc ^= (row[j] & pbit(v, j));
    return acc;
}

/* One term's exact numerator (zx_eval.hpp:101-165), no prefactor power2. */
static void eval_term(const ksim_graph_desc *g, int t_g, const pvec_t *v, zw_t *out, int64_t *out_pw)
{
    const int P = g->P;
    zw_t acc = {1, 0, 0, 0};
    int64_t pw = 0;
    /* NodePhases: prod (1 + w^((4 par + phi) mod 8)), renormalised per factor */
    {
        int cnt = g->np_counts[t_g];
        for (int t = 0; t < cnt; ++t) {
            const uint8_t *row = g->np_params + ((size_t)t_g * g->Tnp + t) * (size_t)P;
            int par = parity_row(row, P, v);
            int k = (4 * par + g->np_phases[(size_t)t_g * g->Tnp + t]) & 7;
            zw_t u = zunit(k);
            u.a += 1;
            acc = zmul(acc, u);
            zreduce(&acc, &pw);
        }
    }
    /* HalfPiPhases: w^(sum par*coeff mod 8) over the full padded width */
    {
        int tot = 0;
        for (int t = 0; t < g->Thp; ++t) {
            const uint8_t *row = g->hp_params + ((size_t)t_g * g->Thp + t) * (size_t)P;
            int par = parity_row(row, P, v);
            tot += (par * g->hp_coeffs[(size_t)t_g * g->Thp + t]) & 7;
        }
        acc = zmul(acc, zunit(tot & 7));
        zreduce(&acc, &pw);
    }
    /* PiProducts: (-1)^(xor psi*phi), psi/phi = const xor parity */
    {
        int e = 0;
        for (int t = 0; t < g->Tpp; ++t) {
            size_t ci = (size_t)t_g * g->Tpp + t;
            int psi = (g->pp_psi_c[ci] + parity_row(g->pp_psi_p + ci * (size_t)P, P, v)) & 1;
            int phi = (g->pp_phi_c[ci] + parity_row(g->pp_phi_p + ci * (size_t)P, P, v)) & 1;
            e ^= (psi & phi);
        }
        if (e) { acc.a = -acc.a; acc.b = -acc.b; acc.c = -acc.c; acc.d = -acc.d; }
    }
    /* PhasePairs: prod (1 + w^a + w^b - w^(a+b)), renormalised per factor */
    {
        int cnt = g->ph_counts[t_g];
        for (int t = 0; t < cnt; ++t) {
            size_t ci = (size_t)t_g * g->Tph + t;
            int al = (g->ph_alpha[ci] + 4 * parity_row(g->ph_alpha_p + ci * (size_t)P, P, v)) & 7;
            int be = (g->ph_beta[ci] + 4 * parity_row(g->ph_beta_p + ci * (size_t)P, P, v)) & 7;
            zw_t u = zunit(al), w = zunit(be), x = zunit((al + be) & 7);
            zw_t term = {1 + u.a + w.a - x.a, u.b + w.b - x.b, u.c + w.c - x.c, u.d + w.d - x.d};
            acc = zmul(acc, term);
            zreduce(&acc, &pw);
        }
    }
    /* prefactor: w^idx (no renormalisation), then the exact floatfactor */
    acc = zmul(acc, zunit(g->pf_phase_idx[t_g] & 7));
    {
        const int32_t *ff = g->pf_floatfactor + (size_t)t_g * 4;
        zw_t f = {ff[0], ff[1], ff[2], ff[3]};
        acc = zmul(acc, f);
        zreduce(&acc, &pw);
    }
    *out = acc;
    *out_pw = pw;
}

static const double SQ = 0.70710678118654752440; /* cos(pi/4) */

/* Complex amplitude of one graph (zx_eval.hpp:166-181): per-term complex cast,
 * x 2^(pw + power2), optional approximate factor, sequential sum over g. */
static void eval_graph(const ksim_graph_desc *g, const pvec_t *v, double *out_re, double *out_im)
{
    double sum_re = 0.0, sum_im = 0.0;
    for (int t = 0; t < g->G; ++t) {
        zw_t acc;
        int64_t pw;
        eval_term(g, t, v, &acc, &pw);
        double re = (double)acc.a + ((double)acc.b + (double)acc.d) * SQ;
        double im = (double)acc.c + ((double)acc.b - (double)acc.d) * SQ;
        double scale = exp2((double)(pw + g->pf_power2[t]));
        re *= scale;
        im *= scale;
        if (g->pf_has_approx) {
            double ar = (double)g->pf_approx_f32[2 * t];
            double ai = (double)g->pf_approx_f32[2 * t + 1];
            double r2 = re * ar - im * ai;
            im = re * ai + im * ar;
            re = r2;
        }
        sum_re += re;
        sum_im += im;
    }
    *out_re = sum_re;
    *out_im = sum_im;
}

/* ---- uniform streams ---------------------------------------------------- */

void oracle_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4])
{
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c0 = n0; c1 = (uint32_t)p1; c2 = n2; c3 = (uint32_t)p0;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

double oracle_philox_uniform(uint64_t seed, uint64_t shot, uint32_t output)
{
    uint32_t ctr[4] = {(uint32_t)shot, (uint32_t)(shot >> 32), output, 0u};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t x[4];
    oracle_philox4x32_10(ctr, key, x);
    uint64_t bits = ((uint64_t)x[1] << 32) | x[0];
    return (double)(bits >> 11) * (1.0 / 9007199254740992.0);
}

static inline uint64_t xorshift_init(uint64_t seed, uint64_t s)
{
    uint64_t r = seed ^ (s * 0x9e3779b97f4a7c15ULL);
    r ^= r >> 30;
    r *= 0xbf58476d1ce4e5b9ULL;
    r ^= r >> 27;
    return r ? r : 1ULL;
}

static inline double xorshift_uniform(uint64_t *s)
{
    *s ^= *s << 13;
    *s ^= *s >> 7;
    *s ^= *s << 17;
    return (double)(*s >> 11) * (1.0 / (double)(1ULL << 53));
}

/* ---- entry points -------------------------------------------------------- */

/* Sample one component (kokkos_sim.cpp:188-241 semantics).  f_sel (B,F),
 * out (B, max(n_out,1)).  amp (nullable): (B, n_out+1) |A_k|.  Shot s uses
 * stream index shot_offset + s.  n_threads <= 0: OpenMP default. */
int oracle_sample(const ksim_graph_desc *graphs, int n_graphs, int F, const uint8_t *f_sel,
                  int64_t B, int64_t shot_offset, uint64_t seed, int rng_mode,
                  uint8_t *out, double *amp, int n_threads)
{
    if (n_graphs < 1 || F < 0 || B < 0) return 1;
    const int n_out = n_graphs - 1;
    const int ncol = n_out > 1 ? n_out : 1;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#else
    (void)n_threads;
#endif
#pragma omp parallel
    {
        uint8_t *m = (uint8_t *)calloc((size_t)ncol, 1);
#pragma omp for schedule(dynamic, 16)
        for (int64_t s = 0; s < B; ++s) {
            memset(m, 0, (size_t)ncol);
            const uint64_t gs = (uint64_t)(shot_offset + s);
            uint64_t rng = xorshift_init(seed, gs);
            pvec_t v = {f_sel + (size_t)s * (size_t)F, m, F, 0, 0};
            double re, im;
            eval_graph(&graphs[0], &v, &re, &im);
            double prev = sqrt(re * re + im * im);
            if (amp) amp[(size_t)s * (size_t)(n_out + 1)] = prev;
            for (int i = 0; i < n_out; ++i) {
                v.nm = i;
                v.trying = 1;
                eval_graph(&graphs[i + 1], &v, &re, &im);
                double p1 = sqrt(re * re + im * im);
                if (amp) amp[(size_t)s * (size_t)(n_out + 1) + 1 + i] = p1;
                double u = rng_mode == KSIM_RNG_PHILOX ? oracle_philox_uniform(seed, gs, (uint32_t)i)
                                                       : xorshift_uniform(&rng);
                int bit = u < (p1 / prev) ? 1 : 0;
                m[i] = (uint8_t)bit;
                prev = bit ? p1 : (prev - p1);
            }
            memcpy(out + (size_t)s * (size_t)ncol, m, (size_t)ncol);
        }
        free(m);
    }
    return 0;
}

/* Complex amplitude of graph gi on explicit parameter rows (kokkos_sim.cpp:157-185:
 * all P columns come through the f view, no sampled bits, trying = 0). */
int oracle_eval(const ksim_graph_desc *graphs, int n_graphs, int gi, const uint8_t *params,
                int64_t B, int64_t P, double *out_re_im)
{
    if (gi < 0 || gi >= n_graphs || B < 0 || P < 0) return 1;
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < B; ++s) {
        pvec_t v = {params + (size_t)s * (size_t)P, NULL, (int)P, 0, 0};
        eval_graph(&graphs[gi], &v, &out_re_im[2 * s], &out_re_im[2 * s + 1]);
    }
    return 0;
}

/* Per-term numerators (a,b,c,d,pw) of graph gi: out (B, G, 5). */
int oracle_eval_terms(const ksim_graph_desc *graphs, int n_graphs, int gi, const uint8_t *params,
                      int64_t B, int64_t P, int64_t *out)
{
    if (gi < 0 || gi >= n_graphs || B < 0 || P < 0) return 1;
    const ksim_graph_desc *g = &graphs[gi];
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < B; ++s) {
        pvec_t v = {params + (size_t)s * (size_t)P, NULL, (int)P, 0, 0};
        for (int t = 0; t < g->G; ++t) {
            zw_t acc;
            int64_t pw;
            eval_term(g, t, &v, &acc, &pw);
            int64_t *o = out + ((size_t)s * g->G + t) * 5;
            o[0] = acc.a; o[1] = acc.b; o[2] = acc.c; o[3] = acc.d; o[4] = pw;
        }
    }
    return 0;
}

/* exp2 of an integer, as the reference's complex cast calls it. */
double oracle_exp2_int(int64_t n) { return exp2((double)n); }

int oracle_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ---- noise draw ----------------------------------------------------------
 * CPU restatement of the device noise draw (ksim_b200/csrc/noise.cu), the
 * checker for it.  The model follows ChannelSampler (compile/channels.py:
 * 480-622): channels with p_fire = 1 - probs[0] <= 1e-15 never fire;
 * channels over identical error-bit patterns (same bit count, same
 * error_transform columns in order) are merged by XOR convolution, in order
 * of first appearance; the conditional CDF is cumsum(probs[1:] / p_fire)
 * normalised by its last entry.  The merged channels are ordered by p_fire
 * (descending, ties in merged order) and cut into runs of equal p_fire, each
 * with the table T_k = floor((1 - p)^k 2^32), k = 1.. (while > 0, at most the
 * run's length).  Per shot, a stream of 32-bit draws (Philox4x32-10, key =
 * seed, counter = (shot lo, shot hi, block, 'NOIS'), four words a block, in
 * order) drives, per run, jumps from channel j to j + 1 + #{k : u < T_k};
 * a channel jumped to fires with the first outcome o whose threshold
 * floor(cdf_o 2^32) exceeds the next draw, and its f pattern is XORed in. */
static uint32_t noise_threshold32(double u)
{
    if (!(u > 0.0)) return 0u;
    double t = floor(ldexp(u, 32));
    return t >= 4294967295.0 ? 4294967295u : (uint32_t)t;
}

typedef struct {
    int k;
    double *p;       /* 2^k outcome probabilities */
    uint64_t *bits;  /* k patterns of nw words */
} nz_chan;

typedef struct {
    double p;
    int idx;
} nz_key;

static int nz_cmp(const void *a, const void *b)
{
    const nz_key *x = (const nz_key *)a, *y = (const nz_key *)b;
    if (x->p != y->p) return x->p > y->p ? -1 : 1;
    return x->idx < y->idx ? -1 : x->idx > y->idx ? 1 : 0;
}

typedef struct {
    uint64_t shot, seed;
    uint32_t blk, pos, buf[4];
} nz_stream;

static uint32_t nz_next(nz_stream *st)
{
    if (st->pos == 4) {
        uint32_t ctr[4] = {(uint32_t)st->shot, (uint32_t)(st->shot >> 32), st->blk++, 0x4E4F4953u};
        uint32_t key[2] = {(uint32_t)st->seed, (uint32_t)(st->seed >> 32)};
        oracle_philox4x32_10(ctr, key, st->buf);
        st->pos = 0;
    }
    return st->buf[st->pos++];
}

int oracle_noise_sample(const double *probs, const int32_t *n_bits, int n_channels, const uint8_t *transform,
                        int num_f, int num_e, int64_t B, int64_t shot_offset, uint64_t seed, uint8_t *out)
{
    const int nw = num_f > 0 ? (num_f + 63) / 64 : 1;
    uint64_t *col = (uint64_t *)calloc((size_t)(num_e > 0 ? num_e : 1) * nw, sizeof(uint64_t));
    nz_chan *m = (nz_chan *)calloc((size_t)(n_channels > 0 ? n_channels : 1), sizeof(nz_chan));
    if (!col || !m) return 1;
    for (int fi = 0; fi < num_f; ++fi)
        for (int e = 0; e < num_e; ++e)
            if (transform[(size_t)fi * num_e + e]) col[(size_t)e * nw + fi / 64] |= 1ull << (fi % 64);
    /* drop never-firing channels, merge identical signatures */
    int n_m = 0;
    int64_t po = 0;
    int eo = 0;
    for (int i = 0; i < n_channels; ++i) {
        const int k = n_bits[i];
        const int64_t n = (int64_t)1 << k;
        const double *pr = probs + po;
        const int e0 = eo;
        po += n;
        eo += k;
        if (!(1.0 - pr[0] > 1e-15) || n <= 1) continue;
        int hit = -1;
        for (int j = 0; j < n_m && hit < 0; ++j) {
            if (m[j].k != k) continue;
            int same = 1;
            for (int b = 0; b < k && same; ++b)
                for (int w = 0; w < nw; ++w)
                    if (m[j].bits[(size_t)b * nw + w] != col[(size_t)(e0 + b) * nw + w]) { same = 0; break; }
            if (same) hit = j;
        }
        if (hit >= 0) {
            double *cv = (double *)calloc((size_t)n, sizeof(double));
            for (int64_t a = 0; a < n; ++a)
                for (int64_t b = 0; b < n; ++b) cv[a ^ b] += m[hit].p[a] * pr[b];
            free(m[hit].p);
            m[hit].p = cv;
        } else {
            m[n_m].k = k;
            m[n_m].p = (double *)malloc(sizeof(double) * (size_t)n);
            memcpy(m[n_m].p, pr, sizeof(double) * (size_t)n);
            m[n_m].bits = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(k > 0 ? k : 1) * nw);
            memcpy(m[n_m].bits, col + (size_t)e0 * nw, sizeof(uint64_t) * (size_t)k * nw);
            ++n_m;
        }
    }
    /* order by p_fire, runs, skip tables, CDF thresholds, outcome patterns */
    nz_key *ord = (nz_key *)calloc((size_t)(n_m > 0 ? n_m : 1), sizeof(nz_key));
    int n_live = 0;
    for (int j = 0; j < n_m; ++j)
        if (1.0 - m[j].p[0] > 1e-15) {
            ord[n_live].p = 1.0 - m[j].p[0];
            ord[n_live].idx = j;
            ++n_live;
        }
    qsort(ord, (size_t)n_live, sizeof(nz_key), nz_cmp);
    int *run_first = (int *)calloc((size_t)(n_live > 0 ? n_live : 1), sizeof(int));
    int *run_n = (int *)calloc((size_t)(n_live > 0 ? n_live : 1), sizeof(int));
    uint32_t **run_tab = (uint32_t **)calloc((size_t)(n_live > 0 ? n_live : 1), sizeof(uint32_t *));
    int *run_len = (int *)calloc((size_t)(n_live > 0 ? n_live : 1), sizeof(int));
    uint32_t **cdf = (uint32_t **)calloc((size_t)(n_live > 0 ? n_live : 1), sizeof(uint32_t *));
    uint64_t **pat = (uint64_t **)calloc((size_t)(n_live > 0 ? n_live : 1), sizeof(uint64_t *));
    int n_runs = 0;
    for (int r0 = 0; r0 < n_live;) {
        int r1 = r0;
        while (r1 < n_live && ord[r1].p == ord[r0].p) ++r1;
        run_first[n_runs] = r0;
        run_n[n_runs] = r1 - r0;
        run_tab[n_runs] = (uint32_t *)calloc((size_t)(r1 - r0), sizeof(uint32_t));
        const double q = 1.0 - ord[r0].p;
        double t = 1.0;
        int len = 0;
        for (int k = 1; k <= r1 - r0; ++k) {
            t *= q;
            const uint32_t thr = noise_threshold32(t);
            if (thr == 0) break;
            run_tab[n_runs][len++] = thr;
        }
        run_len[n_runs] = len;
        for (int x = r0; x < r1; ++x) {
            const nz_chan *c = &m[ord[x].idx];
            const int64_t n = (int64_t)1 << c->k;
            const double p_fire = ord[x].p;
            double *cum = (double *)calloc((size_t)n, sizeof(double));
            double run = 0;
            for (int64_t o = 1; o < n; ++o) {
                run += (c->p[o] > 0.0 ? c->p[o] : 0.0) / p_fire;
                cum[o - 1] = run;
            }
            cdf[x] = (uint32_t *)calloc((size_t)n, sizeof(uint32_t));
            for (int64_t o = 0; o + 1 < n - 1; ++o) cdf[x][o] = noise_threshold32(cum[o] / cum[n - 2]);
            free(cum);
            pat[x] = (uint64_t *)calloc((size_t)n * nw, sizeof(uint64_t));
            for (int64_t o = 1; o < n; ++o)
                for (int b = 0; b < c->k; ++b)
                    if ((o >> b) & 1)
                        for (int w = 0; w < nw; ++w) pat[x][(size_t)(o - 1) * nw + w] ^= c->bits[(size_t)b * nw + w];
        }
        ++n_runs;
        r0 = r1;
    }
    uint64_t *acc = (uint64_t *)calloc((size_t)nw, sizeof(uint64_t));
    for (int64_t s = 0; s < B; ++s) {
        nz_stream st = {(uint64_t)(shot_offset + s), seed, 0u, 4u, {0, 0, 0, 0}};
        memset(acc, 0, sizeof(uint64_t) * (size_t)nw);
        for (int r = 0; r < n_runs; ++r) {
            int64_t j = -1;
            for (;;) {
                const uint32_t u = nz_next(&st);
                int64_t kk = 0;
                while (kk < run_len[r] && u < run_tab[r][kk]) ++kk; /* #{k : u < T_k}, T decreasing */
                j += kk + 1;
                if (j >= run_n[r]) break;
                const int x = run_first[r] + (int)j;
                const int64_t n_out = ((int64_t)1 << m[ord[x].idx].k) - 1;
                const uint32_t v = nz_next(&st);
                int64_t o = 0;
                while (o + 1 < n_out && v >= cdf[x][o]) ++o;
                for (int w = 0; w < nw; ++w) acc[w] ^= pat[x][(size_t)o * nw + w];
            }
        }
        for (int fi = 0; fi < num_f; ++fi) out[s * num_f + fi] = (uint8_t)((acc[fi / 64] >> (fi % 64)) & 1u);
    }
    for (int x = 0; x < n_live; ++x) { free(cdf[x]); free(pat[x]); }
    for (int r = 0; r < n_runs; ++r) free(run_tab[r]);
    for (int j = 0; j < n_m; ++j) { free(m[j].p); free(m[j].bits); }
    free(col); free(m); free(ord); free(run_first); free(run_n); free(run_tab); free(run_len);
    free(cdf); free(pat); free(acc);
    return 0;
}
