// image.cpp — validation and packing of a component into the device image.
//
// Input: the reference's per-graph arrays (sampler.py:21-43 dict layout,
// kokkos_sim.cpp:91-129 field set).  Output: one byte image
//   [GraphDir x n_graphs][term stream of graph 0][term stream of graph 1]...
// Each term record (16-byte aligned) starts with a 96-byte header:
//   u32 n_np | n_hp<<16, u32 n_pp | n_ph<<16, u32 pf_idx | flags<<16,
//   i32 power2, i32 floatfactor[4], u32 n0 | n2<<16, u32 n1 | n3<<16 (the
//   NodePhases columns per rotation class), i32 H (the block's halvings),
//   u32 record bytes, u64 C[4] (the block's all-plus product / 2^H, mod
//   2^64), u32 nb (parity blocks), and for a fast term its layout: u16
//   offsets / 16 of the PhasePairs tables, step tables, lambda table and
//   parity blocks, u16 first PhasePairs row, u16 nu0 | constants' offset / 16
//   << 2 (zeros for an exact term),
// then [f64 approx re, im], then the body.  A fast term's body is its parity
// rows (layout: zring.cuh).  An exact (TF_SLOW) term's body is the columns
// in the reference's order, each the parameter masks as W 64-bit words (bit j
// = param j; the top bit of word W-1 is the constant 1 of the parameter
// vector, set in a mask when the column's constant is 1) and one constant
// word:
//   NodePhases  [mask W][phase]                              (count = np_counts[g])
//   HalfPi      [mask W][coeff & 7]                          (zero coeffs dropped)
//   PiProducts  [psi W][phi W][psi_c | phi_c<<1]             (identically-zero dropped)
//   PhasePairs  [alpha W][beta W][ja | K<<2 | jb<<3 | jg<<5] (count = ph_counts[g])
// Dropped columns contribute nothing in the reference either (a zero HalfPi
// coefficient adds 0 to the phase sum; a PiProducts column whose psi or phi is
// identically 0 adds psi*phi = 0).
#include "image.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <map>

#include "zring.cuh"

namespace ksim {

namespace {

constexpr int kWords[] = {1, 2, 3, 4, 5, 6, 8, 10, 12, 16};

void put32(std::vector<uint8_t> &b, uint32_t v)
{
    uint8_t t[4];
    std::memcpy(t, &v, 4);
    b.insert(b.end(), t, t + 4);
}
void put64(std::vector<uint8_t> &b, uint64_t v)
{
    uint8_t t[8];
    std::memcpy(t, &v, 8);
    b.insert(b.end(), t, t + 8);
}

// sigma_k(z) for the embedding w -> e^{i k pi/4}.
std::complex<double> embed(const int64_t z[4], int k)
{
    const double th = k * M_PI / 4;
    const std::complex<double> w(std::cos(th), std::sin(th));
    return (double)z[0] + (double)z[1] * w + (double)z[2] * (w * w) + (double)z[3] * std::conj(w);
}

double max_embed(const int64_t z[4])
{
    double m = 0;
    for (int k = 1; k < 8; k += 2) m = std::max(m, std::abs(embed(z, k)));
    return m;
}

void unit(int k, int64_t out[4])
{
    static const int64_t t[8][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, -1},
                                    {-1, 0, 0, 0}, {0, -1, 0, 0}, {0, 0, -1, 0}, {0, 0, 0, 1}};
    for (int i = 0; i < 4; ++i) out[i] = t[k & 7][i];
}

// 1 + w^a + w^b - w^(a+b)
void phase_pair(int a, int b, int64_t out[4])
{
    int64_t u[4], v[4], x[4];
    unit(a, u); unit(b, v); unit(a + b, x);
    for (int i = 0; i < 4; ++i) out[i] = u[i] + v[i] - x[i];
    out[0] += 1;
}

struct Bits {
    const uint8_t *row;  // P bytes
};

// Pack one P-byte mask row into W words; false if a byte is neither 0 nor 1.
bool pack_mask(const uint8_t *row, int P, int W, uint64_t *out)
{
    for (int w = 0; w < W; ++w) out[w] = 0;
    for (int j = 0; j < P; ++j) {
        const uint8_t b = row[j];
        if (b > 1) return false;
        out[j >> 6] |= (uint64_t)b << (j & 63);
    }
    return true;
}

bool all_zero(const uint64_t *m, int W)
{
    for (int w = 0; w < W; ++w)
        if (m[w]) return false;
    return true;
}

}  // namespace

// Work model: int32 operations one shot costs for one term / graph in the
// formulation the kernels run (the roofline numerator).  c = 1 on 32-bit
// words (TF_NARROW), 2 on 64-bit words; exact-path terms are costed as the
// reference's step-by-step arithmetic (one Z[w] product = 16 64-bit
// multiplies x 3 + 12 64-bit adds x 2 + renormalisation 12 = 84 per factor,
// and a parity of a W-word mask 3W + 2).
//   fast term, per 32-row parity block (64 shots of a warp share it):
//     row XORs: 32 rows x n_iter x 2 (64-bit xor) / 64 shots = n_iter
//       (n_iter: index slots per row of the block, even)
//     transposes: 2 x 5 rounds x 2 (rotate, select) x 32 lanes / 64 = 10
//     block sums: 4 (and) + 4 (popcount) + 1 (shift) + 4 (accumulate) = 13
//   NodePhases: C * lambda^e, 16 multiply-adds x c_np + 4 (mask) + 2
//   PhasePairs, per pair of columns (an odd last one pairs with 1): 3 (sign
//               bits) + 6 (valuations) + 8 (two halving decisions) + 8 (factor
//               read and unpack) + 16c (product) + 4c + 1 (shift, pw)
//   per term: ff * w^k read 4, floatfactor product 16 (c = 1) or 64 (c = 2),
//             renormalisation 6c, complex value and sum 16
//   per graph: parameter vector 4W + 8, ballot words 4, Bernoulli step 10
double term_work(int W, uint32_t flags, const int n_cls[4], int n_hp, int n_pp, int n_ph, int nb, int sum_iter)
{
    const double par = 3.0 * W + 2.0;
    const int n_np = n_cls[0] + n_cls[1] + n_cls[2] + n_cls[3];
    if (flags & TF_SLOW)
        return 84.0 * (n_np + n_ph + 3) + par * (n_np + n_hp + 2.0 * n_pp + 2.0 * n_ph) + 16.0;
    const double c = (flags & TF_NARROW) ? 1.0 : 2.0;
    const double cn = (flags & (TF_NARROW | TF_HYBRID)) ? 1.0 : 2.0;  // NodePhases words
    double w = (double)sum_iter + 23.0 * nb;
    if (n_cls[1] | n_cls[3]) w += 2.0;  // the block's product read from the term's lambda table
    w += 4.0 * cn;
    w += ((n_ph + 1) / 2) * (3.0 + 5.0 + 8.0 + 8.0 + 16.0 * c + 4.0 * c + 1.0);
    w += 4.0 + (c == 1.0 ? 16.0 : 64.0) + 6.0 * c + 16.0;
    return w;
}

double graph_work(int W) { return 4.0 * W + 8.0 + 4.0 + 10.0; }

int supported_words(int needed)
{
    for (int w : kWords)
        if (w >= needed) return w;
    return -1;
}

uint32_t zw_valuation(const int64_t z[4])
{
    if (!z[0] && !z[1] && !z[2] && !z[3]) return NU_ZERO;
    // z * conj(z) = p + q sqrt2, conj(a,b,c,d) = (a,d,-c,b); N(z) = p^2 - 2 q^2
    typedef __int128 i128;
    const i128 a = z[0], b = z[1], c = z[2], d = z[3];
    const i128 ca = a, cb = d, cc = -c, cd = b;
    const i128 p = a * ca + b * cd - c * cc + d * cb;
    const i128 q = a * cb + b * ca + c * cd + d * cc;
    i128 n = p * p - 2 * q * q;
    if (n < 0) n = -n;
    uint32_t v = 0;
    while (n != 0 && (n & 1) == 0) {
        n >>= 1;
        ++v;
    }
    return v;
}

int build_image(const ksim_graph_desc *gs, int n_graphs, int F, HostImage &img, std::string &err)
{
    if (n_graphs < 1) {
        err = "a component needs at least one graph (the normalisation graph)";
        return KSIM_ERR_INVALID_ARGUMENT;
    }
    if (F < 0) {
        err = "num_f must be >= 0";
        return KSIM_ERR_INVALID_ARGUMENT;
    }
    if (!gs) {
        err = "graphs is NULL";
        return KSIM_ERR_INVALID_ARGUMENT;
    }
    const int n_out = n_graphs - 1;
    int64_t need_bits = (int64_t)F + n_out;
    for (int k = 0; k < n_graphs; ++k) {
        const ksim_graph_desc &g = gs[k];
        if (g.G < 0 || g.P < 0 || g.Tnp < 0 || g.Thp < 0 || g.Tpp < 0 || g.Tph < 0) {
            err = "graph " + std::to_string(k) + ": negative dimension";
            return KSIM_ERR_MALFORMED_PROGRAM;
        }
        need_bits = std::max<int64_t>(need_bits, g.P);
    }
    // one more bit than the parameters: the top bit of the vector is the
    // constant 1 that folds each column's constant into its parity
    const int W = supported_words((int)std::max<int64_t>(1, (need_bits + 1 + 63) / 64));
    if (W < 0 || need_bits + 1 > 64 * 16) {
        err = "parameter vector of " + std::to_string(need_bits) +
              " bits exceeds the 1023 this build supports";
        return KSIM_ERR_UNSUPPORTED;
    }
    const uint64_t one_bit = 1ull << 63;  // in word W - 1
    const int R1 = rec1_words(W), R2 = rec2_words(W);

    img = HostImage();
    img.n_graphs = n_graphs;
    img.F = F;
    img.n_out = n_out;
    img.W = W;
    img.gdir.resize(n_graphs);
    img.term_off.resize(n_graphs);
    std::vector<uint8_t> &out = img.bytes;
    out.resize(sizeof(GraphDir) * (size_t)n_graphs, 0);

    std::vector<uint64_t> mask(2 * W);
    std::vector<uint8_t> zero_row;

    for (int k = 0; k < n_graphs; ++k) {
        const ksim_graph_desc &g = gs[k];
        const int G = g.G, P = g.P;
        const std::string gname = "graph " + std::to_string(k);
        auto need = [&](const void *p, int64_t n, const char *name) -> bool {
            if (n > 0 && !p) {
                err = gname + ": " + name + " is NULL but has " + std::to_string(n) + " elements";
                return false;
            }
            return true;
        };
        if (!need(g.np_phases, (int64_t)G * g.Tnp, "np_phases") ||
            !need(g.np_params, (int64_t)G * g.Tnp * P, "np_params") ||
            !need(g.np_counts, G, "np_counts") || !need(g.hp_coeffs, (int64_t)G * g.Thp, "hp_coeffs") ||
            !need(g.hp_params, (int64_t)G * g.Thp * P, "hp_params") ||
            !need(g.pp_psi_c, (int64_t)G * g.Tpp, "pp_psi_c") ||
            !need(g.pp_psi_p, (int64_t)G * g.Tpp * P, "pp_psi_p") ||
            !need(g.pp_phi_c, (int64_t)G * g.Tpp, "pp_phi_c") ||
            !need(g.pp_phi_p, (int64_t)G * g.Tpp * P, "pp_phi_p") ||
            !need(g.ph_alpha, (int64_t)G * g.Tph, "ph_alpha") ||
            !need(g.ph_alpha_p, (int64_t)G * g.Tph * P, "ph_alpha_p") ||
            !need(g.ph_beta, (int64_t)G * g.Tph, "ph_beta") ||
            !need(g.ph_beta_p, (int64_t)G * g.Tph * P, "ph_beta_p") ||
            !need(g.ph_counts, G, "ph_counts") || !need(g.pf_phase_idx, G, "pf_phase_idx") ||
            !need(g.pf_floatfactor, 4 * (int64_t)G, "pf_floatfactor") ||
            !need(g.pf_power2, G, "pf_power2") ||
            !need(g.pf_approx_f32, g.pf_has_approx ? 2 * (int64_t)G : 0, "pf_approx_f32"))
            return KSIM_ERR_MALFORMED_PROGRAM;

        GraphDir &gd = img.gdir[k];
        gd.G = G;
        gd.P = P;
        gd.stream_off = (int64_t)out.size();
        std::vector<int64_t> &toff = img.term_off[k];
        toff.reserve(G + 1);

        for (int t = 0; t < G; ++t) {
            const int64_t start = (int64_t)out.size();
            toff.push_back(start);
            // counts: the reference loops t < count, so a negative count is an
            // empty loop; a count above the padded width would read another
            // term's rows and is rejected.
            int cnp = std::max(0, g.np_counts[t]);
            int cph = std::max(0, g.ph_counts[t]);
            if (cnp > g.Tnp || cph > g.Tph) {
                err = gname + ": term " + std::to_string(t) + " count exceeds the padded width";
                return KSIM_ERR_MALFORMED_PROGRAM;
            }
            std::vector<uint8_t> rec;  // column records of this term (exact path)
            struct Row { std::vector<uint64_t> m; uint32_t c; };
            std::vector<Row> hp_rows, pair_rows, ph_rows;  // parity rows (fast paths)
            // Bounds, as log2 of max_k |sigma_k(z)| (>= every coefficient):
            //   ref_max: every value the reference's step-by-step arithmetic
            //     holds (its int64 must not wrap, else the term takes the exact
            //     path, which wraps like it);
            //   fast_max: every value the fast path must know exactly — after
            //     each PhasePairs factor (the evenness test and halving) and
            //     at the end; everything between is ring arithmetic that may
            //     wrap.  The NodePhases result itself must be exact only
            //     where it is widened (the hybrid path).
            double L = 0;  // z starts at 1
            double ref_max = 0, fast_max = 0;
            const double kLim = 62.0 - 1e-9;
            bool unsafe = false;
            // NodePhases.  A column's mask carries the constant bit iff bit 2
            // of its phase is set, so its parity is the sign of w^(4 par):
            // factor = 1 + (-1)^parity w^(phase & 3).  Every factor has
            // valuation <= 2 and the reference halves at most once per
            // factor, so the block's result is order-independent:
            // prod / 2^floor(sum nu / 4).  Fast terms therefore keep their
            // columns grouped by rotation class (j = 0, 2, 1, 3) and reduce
            // each class to a sign count (zring.cuh); exact terms keep the
            // reference's order.
            struct NpCol { uint32_t phase; std::vector<uint64_t> m; };
            std::vector<NpCol> npc((size_t)cnp);
            for (int c = 0; c < cnp; ++c) {
                const size_t ci = (size_t)t * g.Tnp + c;
                if (!pack_mask(g.np_params + ci * P, P, W, mask.data())) {
                    err = gname + ": np_params holds a byte other than 0/1";
                    return KSIM_ERR_MALFORMED_PROGRAM;
                }
                npc[c].phase = g.np_phases[ci] & 7u;
                npc[c].m.assign(mask.begin(), mask.begin() + W);
                if (npc[c].phase & 4u) npc[c].m[W - 1] |= one_bit;
            }
            static const int kClassRank[4] = {0, 2, 1, 3};  // j = 0, 1, 2, 3 -> run position
            std::vector<int> order((size_t)cnp);
            for (int c = 0; c < cnp; ++c) order[c] = c;
            std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
                return kClassRank[npc[a].phase & 3u] < kClassRank[npc[b].phase & 3u];
            });
            int n_cls[4] = {0, 0, 0, 0};
            for (int c = 0; c < cnp; ++c) ++n_cls[npc[c].phase & 3u];
            // A term whose factor 2 / 0 column yields 0 keeps the pw the
            // reference had at that column: its earlier factor-2 columns plus
            // the halvings before it in the reference's order (dead_pw, stored
            // in the column word; class-0 columns keep their relative order).
            std::vector<uint32_t> dead_pw((size_t)cnp, 0);
            {
                uint32_t cum = 0, n_two = 0;
                for (int c = 0; c < cnp; ++c) {
                    const uint32_t j = npc[c].phase & 3u;
                    dead_pw[c] = n_two + cum / 4;
                    if (j) cum += (j & 1u) ? 1u : 2u;
                    else ++n_two;
                }
            }
            // Bound and halving points of the block in run order; C is the
            // all-plus product with the same halvings (class 0 contributes
            // 2 / 2 = 1).
            std::vector<uint32_t> np_red((size_t)cnp, 0);  // halving flag, by run position
            uint32_t nu = 0;
            __int128 C[4] = {1, 0, 0, 0};
            bool c_ok = true;
            for (int r = 0; r < cnp; ++r) {
                const uint32_t j = npc[order[r]].phase & 3u;
                if (j != 0) {
                    nu += (j & 1u) ? 1u : 2u;
                    L += (j & 1u) ? std::log2(2.0 * std::cos(M_PI / 8)) : 0.5;
                    // C *= 1 + w^j: w = (0,1,0,0), i = (0,0,1,0), w^3 = (0,0,0,-1)
                    const __int128 a = C[0], b = C[1], c = C[2], d = C[3];
                    if (j == 1) { C[0] = a + d; C[1] = b + a; C[2] = c + b; C[3] = d - c; }
                    else if (j == 2) { C[0] = a - c; C[1] = b + d; C[2] = c + a; C[3] = d - b; }
                    else { C[0] = a - b; C[1] = b - c; C[2] = c + d; C[3] = d - a; }
                    if (nu >= 4) {
                        nu -= 4;
                        np_red[r] = 1;
                        L -= 1.0;
                        for (int k = 0; k < 4; ++k) {
                            if (C[k] & 1) c_ok = false;
                            C[k] >>= 1;
                        }
                    }
                    for (int k = 0; k < 4; ++k)
                        if (C[k] > ((__int128)1 << 100) || C[k] < -((__int128)1 << 100)) c_ok = false;
                }
            }
            const int n_np = cnp;
            const int32_t np_halvings = n_cls[0] + (int32_t)std::count(np_red.begin(), np_red.end(), 1u);
            // The reference runs the block in its own order.  Each factor adds
            // log|f| >= nu / 4 to the bound (odd j: 0.89 >= 0.25; j = 2: 0.5;
            // j = 0: 1), so in any order a value after a factor is below
            // 2^(S + 0.75) with S = sum (log|f| - nu / 4) over all the block's
            // factors, and the factor-2 transient (2z before its halving)
            // below 2^(S + 1.75).
            const double L_np = L;  // the block's result
            if (cnp > 0) ref_max = std::max(ref_max, L_np - (double)nu / 4.0 + 1.75);
            ref_max = std::max(ref_max, L_np);
            // PhasePairs: the bound per valuation of z ((1 - w)-adic; the
            // block's result has nu = the leftover above, for every shot
            // whose term survives)
            std::map<uint32_t, double> ph_state;  // the reference's steps
            ph_state[nu] = L_np;
            std::vector<std::pair<uint32_t, uint32_t>> ph_j;  // rotation classes (ja, jb) per column
            // HalfPi
            int n_hp = 0;
            for (int c = 0; c < g.Thp; ++c) {
                const size_t ci = (size_t)t * g.Thp + c;
                if (!pack_mask(g.hp_params + ci * P, P, W, mask.data())) {
                    err = gname + ": hp_params holds a byte other than 0/1";
                    return KSIM_ERR_MALFORMED_PROGRAM;
                }
                const uint32_t coeff = g.hp_coeffs[ci] & 7u;
                if (coeff == 0 || all_zero(mask.data(), W)) continue;
                hp_rows.push_back({std::vector<uint64_t>(mask.begin(), mask.begin() + W), coeff});
                for (int w = 0; w < W; ++w) put64(rec, mask[w]);
                put64(rec, coeff);
                for (int w = W + 1; w < R1; ++w) put64(rec, 0);
                ++n_hp;
            }
            // PiProducts
            int n_pp = 0;
            for (int c = 0; c < g.Tpp; ++c) {
                const size_t ci = (size_t)t * g.Tpp + c;
                if (!pack_mask(g.pp_psi_p + ci * P, P, W, mask.data()) ||
                    !pack_mask(g.pp_phi_p + ci * P, P, W, mask.data() + W)) {
                    err = gname + ": pp params hold a byte other than 0/1";
                    return KSIM_ERR_MALFORMED_PROGRAM;
                }
                const uint32_t pc = g.pp_psi_c[ci] & 1u, qc = g.pp_phi_c[ci] & 1u;
                const bool psi0 = pc == 0 && all_zero(mask.data(), W);
                const bool phi0 = qc == 0 && all_zero(mask.data() + W, W);
                if (psi0 || phi0) continue;
                // constants folded into the parities: psi = parity(psi mask), phi likewise
                if (pc) mask[W - 1] |= one_bit;
                if (qc) mask[2 * W - 1] |= one_bit;
                pair_rows.push_back({std::vector<uint64_t>(mask.begin(), mask.begin() + W), 0});
                pair_rows.push_back({std::vector<uint64_t>(mask.begin() + W, mask.begin() + 2 * W), 0});
                for (int w = 0; w < 2 * W; ++w) put64(rec, mask[w]);
                put64(rec, pc | (qc << 1));
                for (int w = 2 * W + 1; w < R2; ++w) put64(rec, 0);
                ++n_pp;
            }
            // PhasePairs
            int n_ph = 0;
            for (int c = 0; c < cph; ++c) {
                const size_t ci = (size_t)t * g.Tph + c;
                if (!pack_mask(g.ph_alpha_p + ci * P, P, W, mask.data()) ||
                    !pack_mask(g.ph_beta_p + ci * P, P, W, mask.data() + W)) {
                    err = gname + ": ph params hold a byte other than 0/1";
                    return KSIM_ERR_MALFORMED_PROGRAM;
                }
                const uint32_t ac = g.ph_alpha[ci] & 7u, bc = g.ph_beta[ci] & 7u, gc = (ac + bc) & 7u;
                const uint32_t a2 = ac >> 2, b2 = bc >> 2;
                // the masks carry bit 2 of alpha / beta in the constant bit, so
                // pa' = pa ^ a2 and pb' = pb ^ b2 are the signs of the w^a and
                // w^b copies; the -w^(a+b) copy's sign is K ^ pa' ^ pb'
                if (a2) mask[W - 1] |= one_bit;
                if (b2) mask[2 * W - 1] |= one_bit;
                const uint32_t K = ((gc >> 2) ^ 1u ^ a2 ^ b2) & 1u;
                uint64_t cw = (ac & 3u) | (K << 2) | ((bc & 3u) << 3) | ((gc & 3u) << 5);
                // bound through the factor for each valuation state: the value
                // after it is an exact point; the reference then halves once
                // iff nu >= 4 (a zero factor ends the term)
                std::map<uint32_t, double> next;
                for (uint32_t combo = 0; combo < 4; ++combo) {  // combo = raw pa | pb << 1
                    int64_t f[4];
                    phase_pair((int)(ac ^ ((combo & 1u) << 2)), (int)(bc ^ ((combo >> 1) << 2)), f);
                    const uint32_t v = zw_valuation(f);
                    if (v == NU_ZERO) continue;
                    const double lf = std::log2(max_embed(f)) + 1e-12;
                    for (const auto &sv : ph_state) {
                        double x = sv.second + lf;
                        ref_max = std::max(ref_max, x);
                        uint32_t s1 = sv.first + v;
                        if (s1 >= 4) {
                            s1 -= 4;
                            x -= 1.0;
                        }
                        auto it = next.find(s1);
                        if (it == next.end() || it->second < x) next[s1] = x;
                    }
                }
                ph_state.swap(next);
                ph_j.push_back({ac & 3u, bc & 3u});
                ph_rows.push_back({std::vector<uint64_t>(mask.begin(), mask.begin() + W), (uint32_t)cw});
                ph_rows.push_back({std::vector<uint64_t>(mask.begin() + W, mask.begin() + 2 * W), 0});
                for (int w = 0; w < 2 * W; ++w) put64(rec, mask[w]);
                put64(rec, cw);
                for (int w = 2 * W + 1; w < R2; ++w) put64(rec, 0);
                ++n_ph;
            }
            // prefactor
            const int32_t *ff = g.pf_floatfactor + 4 * (size_t)t;
            const int64_t ff64[4] = {ff[0], ff[1], ff[2], ff[3]};
            const double S = std::fabs((double)ff[0]) + std::fabs((double)ff[1]) +
                             std::fabs((double)ff[2]) + std::fabs((double)ff[3]);
            if (S > 0)
                for (const auto &sv : ph_state) ref_max = std::max(ref_max, sv.second + std::log2(S) + 1e-12);
            // The fast path runs PhasePairs columns in pairs (zring.cuh): its
            // exact points are the unhalved pair products, then the end.  Pair tables: the 16
            // products F F' by folded signs, and the step table of the pair's
            // halvings (see pair_step below).
            auto ph_factor = [&](size_t col, uint32_t k, int64_t f[4]) {
                phase_pair((int)(ph_j[col].first | ((k & 1u) << 2)), (int)(ph_j[col].second | ((k >> 1) << 2)), f);
            };
            // (an odd last column pairs with the factor 1: valuation 0)
            const size_t n_pair = ((size_t)n_ph + 1) / 2;
            std::vector<uint8_t> pair_tab(64 * n_pair, 0);
            std::vector<uint8_t> pair_step(256 * n_pair, 0);
            bool pair_ok = true;
            auto ph_factor2 = [&](size_t col, uint32_t k, int64_t f[4]) {
                if (col < (size_t)n_ph) {
                    ph_factor(col, k, f);
                } else {
                    f[0] = 1; f[1] = 0; f[2] = 0; f[3] = 0;
                }
            };
            {
                std::map<uint32_t, double> fs;
                fs[nu] = L_np;
                for (size_t q = 0; q < n_pair; ++q) {
                    // step table: entry 16 c + nu (c = the pair's four sign
                    // bits, nu = the valuation of z before the pair, 0..14,
                    // or NU_DEAD: z is zero) holds the pair's halvings
                    // h1 + h2 (bits 0-1) and the state after it (bits 2-5):
                    // the reference halves after a factor iff nu(z) >= 4,
                    // and a zero factor stops the halvings from where it
                    // acts (NU_DEAD absorbs, with no halvings).  A factor can
                    // have nu up to 6, so nu may grow; terms whose reachable
                    // nu leaves 0..14 take the exact path.
                    for (const auto &sv : fs)
                        if (sv.first >= NU_DEAD) pair_ok = false;
                    const uint32_t second = 2 * q + 1 < (size_t)n_ph ? 1u : 0u;
                    for (uint32_t c = 0; c < 16; ++c) {
                        int64_t f1[4], f2[4];
                        ph_factor2(2 * q, c & 3u, f1);
                        ph_factor2(2 * q + 1, c >> 2, f2);
                        const uint32_t v1 = std::min<uint32_t>(zw_valuation(f1), 15u);
                        const uint32_t v2 = std::min<uint32_t>(zw_valuation(f2), 15u);
                        pair_step[256 * q + 16 * c + NU_DEAD] = (uint8_t)(NU_DEAD << 2);
                        for (uint32_t nu0 = 0; nu0 < NU_DEAD; ++nu0) {
                            uint32_t alive = v1 != 15 ? 1u : 0u;
                            uint32_t tt = nu0 + v1;
                            const uint32_t h1 = (tt >= 4 ? 1u : 0u) & alive;
                            alive &= v2 != 15 ? 1u : 0u;
                            tt = tt - 4 * h1 + v2;
                            const uint32_t h2 = (tt >= 4 ? 1u : 0u) & alive & second;
                            const uint32_t nu1 = alive ? tt - 4 * h2 : NU_DEAD;
                            if (alive && nu1 >= NU_DEAD) continue;  // unreachable unless a state above is (then unsafe)
                            pair_step[256 * q + 16 * c + nu0] = (uint8_t)((h1 + h2) | (nu1 << 2));
                        }
                    }
                    std::map<uint32_t, double> next;
                    for (uint32_t c = 0; c < 16; ++c) {
                        int64_t f1[4], f2[4];
                        ph_factor2(2 * q, c & 3u, f1);
                        ph_factor2(2 * q + 1, c >> 2, f2);
                        const Zu a = {(uint64_t)f1[0], (uint64_t)f1[1], (uint64_t)f1[2], (uint64_t)f1[3]};
                        const Zu b = {(uint64_t)f2[0], (uint64_t)f2[1], (uint64_t)f2[2], (uint64_t)f2[3]};
                        const Zu pr = zmul(a, b);
                        const int64_t pc[4] = {(int64_t)pr.a, (int64_t)pr.b, (int64_t)pr.c, (int64_t)pr.d};
                        for (int i = 0; i < 4; ++i) {
                            if (pc[i] < -128 || pc[i] > 127) pair_ok = false;
                            pair_tab[64 * q + 4 * c + (size_t)i] = (uint8_t)(int8_t)pc[i];
                        }
                        const uint32_t v1 = zw_valuation(f1), v2 = zw_valuation(f2);
                        if (v1 == NU_ZERO || v2 == NU_ZERO) continue;
                        const double l12 = std::log2(max_embed(pc)) + 1e-12;
                        for (const auto &sv : fs) {
                            double x = sv.second + l12;
                            fast_max = std::max(fast_max, x);
                            uint32_t s1 = sv.first + v1;
                            if (s1 >= 4) { s1 -= 4; x -= 1.0; }
                            s1 += v2;
                            if (s1 >= 4 && 2 * q + 1 < (size_t)n_ph) { s1 -= 4; x -= 1.0; }
                            auto it = next.find(s1);
                            if (it == next.end() || it->second < x) next[s1] = x;
                        }
                    }
                    fs.swap(next);
                }
                for (const auto &sv : fs)
                    if (sv.first >= NU_DEAD) pair_ok = false;
                if (S > 0)
                    for (const auto &sv : fs) fast_max = std::max(fast_max, sv.second + std::log2(S) + 1e-12);
            }
            if (n_np > 0xFFFF || n_hp > 0xFFFF || n_pp > 0xFFFF || n_ph > 0xFFFF) {
                err = gname + ": a term has more than 65535 columns in one family";
                return KSIM_ERR_UNSUPPORTED;
            }
            // every value the fast path must know exactly is below
            // 2^fast_max; with fast_max <= 30.5 it fits int32 and the term
            // runs on 32-bit words (a fast term's odd classes are far below LAM_MAX columns: each
            // adds about 0.64 to the bound; the check keeps the table lookup
            // in range whatever the bound)
            uint32_t max_dead = 0;
            for (uint32_t d : dead_pw) max_dead = std::max(max_dead, d);
            // (the tabulated ff * w^k negates coefficients: INT32_MIN has no
            // 32-bit negative)
            bool ff_min = false;
            for (int i = 0; i < 4; ++i) ff_min |= ff[i] == INT32_MIN;
            if (ref_max > kLim || fast_max > kLim || !pair_ok || std::max(n_cls[1], n_cls[3]) > LAM_MAX || !c_ok ||
                max_dead > 0xFFFFu || ff_min)
                unsafe = true;
            uint32_t flags = unsafe ? TF_SLOW : (fast_max <= 30.5 ? TF_NARROW : (L_np <= 30.5 ? TF_HYBRID : 0u));
            // the fast paths' parity rows (row order and block masks:
            // zring.cuh); more than NB_MAX blocks of them sends the term to
            // the exact path
            enum : uint32_t { R_P1 = 1, R_P2 = 2, R_P4 = 4, R_E3 = 8, R_E1 = 16, R_PP = 32, R_K0 = 64 };
            std::vector<const std::vector<uint64_t> *> rows;
            std::vector<uint32_t> role;  // mask bits of each row
            const std::vector<uint64_t> zero_row((size_t)W, 0);
            int ph_row0 = 0;
            if (!unsafe) {
                // class-0 NodePhases rows first, in column order: the kill
                // takes the first that fires, and dead_pw is indexed by
                // position.  Then the other NodePhases and the HalfPi rows
                // (single rows) and the PiProducts (psi, phi) pairs (at even
                // positions, so a pair never straddles a block), heaviest
                // first: a block's row loop runs as many index pairs as its
                // row with the most set bits, so grouping the long rows
                // shortens the other blocks' loops.  The PhasePairs pairs
                // follow from a multiple of 4, in column order.
                auto bits = [&](const std::vector<uint64_t> &m) {
                    int n = 0;
                    for (uint64_t x : m) n += __builtin_popcountll(x);
                    return n;
                };
                struct Unit { int weight, first; uint32_t role0; bool pair; const std::vector<uint64_t> *m0; };
                std::vector<Unit> singles, doubles;
                for (int r = 0; r < cnp; ++r) {
                    const uint32_t j = npc[order[r]].phase & 3u;
                    if (j == 0) {
                        rows.push_back(&npc[order[r]].m);
                        role.push_back(R_K0);
                    } else {
                        singles.push_back({bits(npc[order[r]].m), r, R_P2 | R_P4 | (j == 3 ? R_E3 : j == 1 ? R_E1 : 0u),
                                           false, &npc[order[r]].m});
                    }
                }
                for (size_t i = 0; i < hp_rows.size(); ++i) {
                    const Row &h = hp_rows[i];
                    singles.push_back({bits(h.m), cnp + (int)i,
                                       ((h.c & 1u) ? R_P1 : 0u) | ((h.c & 2u) ? R_P2 : 0u) | ((h.c & 4u) ? R_P4 : 0u),
                                       false, &h.m});
                }
                for (size_t i = 0; i + 1 < pair_rows.size(); i += 2)
                    doubles.push_back({std::max(bits(pair_rows[i].m), bits(pair_rows[i + 1].m)), (int)i, R_PP, true,
                                       &pair_rows[i].m});
                auto heavier = [](const Unit &x, const Unit &y) {
                    return x.weight != y.weight ? x.weight > y.weight : x.first < y.first;
                };
                std::sort(singles.begin(), singles.end(), heavier);
                std::sort(doubles.begin(), doubles.end(), heavier);
                size_t si = 0, di = 0;
                auto put_single = [&]() {
                    rows.push_back(singles[si].m0);
                    role.push_back(singles[si].role0);
                    ++si;
                };
                while (si < singles.size() || di < doubles.size()) {
                    const bool take_pair = di < doubles.size() &&
                                           (si == singles.size() || heavier(doubles[di], singles[si]));
                    if (!take_pair) {
                        put_single();
                        continue;
                    }
                    if (rows.size() & 1u) {  // a pair starts at an even position
                        if (si < singles.size()) {
                            put_single();
                        } else {
                            rows.push_back(&zero_row);
                            role.push_back(0u);
                        }
                    }
                    const size_t i = (size_t)doubles[di].first;
                    rows.push_back(&pair_rows[i].m);
                    role.push_back(R_PP);
                    rows.push_back(&pair_rows[i + 1].m);
                    role.push_back(0u);
                    ++di;
                }
                while (rows.size() & 3u) {  // PhasePairs pairs: 4-bit aligned
                    rows.push_back(&zero_row);
                    role.push_back(0u);
                }
                ph_row0 = (int)rows.size();
                for (const Row &q : ph_rows) {
                    rows.push_back(&q.m);
                    role.push_back(0u);
                }
                if (rows.size() > (size_t)32 * NB_MAX) unsafe = true;
            }
            if (unsafe) flags = TF_SLOW;
            if (!unsafe) {
                // the scales 2^(pw + power2) a shot can reach: pw starts at
                // H or at a kill's dead_pw and gains at most two halvings per
                // PhasePairs pair and one renormalisation
                int64_t lo = np_halvings, hi = np_halvings;
                for (int c = 0; c < cnp; ++c)
                    if ((npc[c].phase & 3u) == 0) {
                        lo = std::min<int64_t>(lo, dead_pw[c]);
                        hi = std::max<int64_t>(hi, dead_pw[c]);
                    }
                hi += 2 * (int64_t)((n_ph + 1) / 2) + 1;
                const int64_t p2 = g.pf_power2[t];
                if (p2 + lo >= -1022 && p2 + hi <= 1023) flags |= TF_EXP;
            }
            if (g.pf_has_approx) flags |= TF_APX;
            std::vector<uint8_t> body;  // everything after the header (and approximation)
            uint32_t nb = 0, sum_iter = 0;
            size_t blocks_at = 0;       // where the parity blocks start in body
            if (unsafe) {
                // the reference's column order and layout
                for (int c = 0; c < cnp; ++c) {
                    for (int w = 0; w < W; ++w) put64(body, npc[c].m[w]);
                    put64(body, (uint64_t)npc[c].phase);
                    for (int w = W + 1; w < R1; ++w) put64(body, 0);
                }
                body.insert(body.end(), rec.begin(), rec.end());
            } else {
                // ff * w^(k + phase index), k = 0..7
                {
                    int64_t z[4] = {ff[0], ff[1], ff[2], ff[3]};
                    for (uint32_t r = 0; r < (g.pf_phase_idx[t] & 7u); ++r) {
                        const int64_t a = z[0], b = z[1], c = z[2], d = z[3];
                        z[0] = d; z[1] = a; z[2] = b; z[3] = -c;  // times w
                    }
                    for (int k = 0; k < 8; ++k) {
                        for (int i = 0; i < 4; ++i) put32(body, (uint32_t)(int32_t)z[i]);
                        const int64_t a = z[0], b = z[1], c = z[2], d = z[3];
                        z[0] = d; z[1] = a; z[2] = b; z[3] = -c;
                    }
                }
                for (int r = 0; r < cnp; ++r)
                    if ((npc[order[r]].phase & 3u) == 0) {
                        const uint32_t d = dead_pw[order[r]];
                        body.push_back((uint8_t)(d & 0xFFu));
                        body.push_back((uint8_t)(d >> 8));
                    }
                while (body.size() & 15u) body.push_back(0);
                body.insert(body.end(), pair_tab.begin(), pair_tab.end());
                body.insert(body.end(), pair_step.begin(), pair_step.end());
                // NodePhases with class-1 / class-3 columns: C lambda^e for
                // e = -n1 .. n3 (mod 2^64; the low words on the 32-bit
                // NodePhases paths), so a shot reads its block's product by
                // its lambda count instead of multiplying
                if (n_cls[1] | n_cls[3]) {
                    const bool np32 = (flags & (TF_NARROW | TF_HYBRID)) != 0;
                    const Zu c = {(uint64_t)C[0], (uint64_t)C[1], (uint64_t)C[2], (uint64_t)C[3]};
                    for (int e = -n_cls[1]; e <= n_cls[3]; ++e) {
                        const Zu z = zmul(c, lam_pow(e, uint64_t()));
                        const uint64_t w4[4] = {z.a, z.b, z.c, z.d};
                        for (int k = 0; k < 4; ++k) {
                            if (np32) put32(body, (uint32_t)w4[k]);
                            else put64(body, w4[k]);
                        }
                    }
                }
                while (body.size() & 15u) body.push_back(0);
                blocks_at = body.size();
                nb = (uint32_t)((rows.size() + 31) / 32);
                const uint16_t zero_off = (uint16_t)(8 * 64 * W);
                for (uint32_t b = 0; b < nb; ++b) {
                    std::vector<std::vector<uint16_t>> lists(32);
                    size_t n_iter = 0;  // index slots per row, rounded up to pairs
                    uint32_t masks[7] = {0, 0, 0, 0, 0, 0, 0};
                    for (int r = 0; r < 32; ++r) {
                        const size_t ri = (size_t)b * 32 + (size_t)r;
                        if (ri >= rows.size()) continue;
                        for (int k = 0; k < 7; ++k)
                            if ((role[ri] >> k) & 1u) masks[k] |= 1u << r;
                        const std::vector<uint64_t> &m = *rows[ri];
                        for (int w = 0; w < W; ++w)
                            for (int k = 0; k < 64; ++k)
                                if ((m[w] >> k) & 1u) lists[r].push_back((uint16_t)(8 * (64 * w + k)));
                        n_iter = std::max(n_iter, lists[r].size());
                    }
                    n_iter = (n_iter + 1) & ~size_t(1);
                    sum_iter += (uint32_t)n_iter;
                    put32(body, (uint32_t)(n_iter / 2));
                    for (int k = 0; k < 7; ++k) put32(body, masks[k]);
                    for (size_t i = 0; i < n_iter; i += 2)
                        for (int r = 0; r < 32; ++r) {
                            const uint16_t o0 = i < lists[r].size() ? lists[r][i] : zero_off;
                            const uint16_t o1 = i + 1 < lists[r].size() ? lists[r][i + 1] : zero_off;
                            put32(body, (uint32_t)o0 | ((uint32_t)o1 << 16));
                        }
                }
            }
            const int apx_bytes = g.pf_has_approx ? TERM_APX_BYTES : 0;
            const uint64_t rec_bytes = (uint64_t)TERM_HDR_BYTES + (uint64_t)apx_bytes + body.size();
            if (rec_bytes > 0xFFFFFFFFull) {
                err = gname + ": a term record exceeds 4 GiB";
                return KSIM_ERR_UNSUPPORTED;
            }
            put32(out, (uint32_t)n_np | ((uint32_t)n_hp << 16));
            put32(out, (uint32_t)n_pp | ((uint32_t)n_ph << 16));
            put32(out, (g.pf_phase_idx[t] & 7u) | (flags << 16));
            put32(out, (uint32_t)g.pf_power2[t]);
            for (int i = 0; i < 4; ++i) put32(out, (uint32_t)ff[i]);
            // NodePhases class counts in run order (j = 0, 2, 1, 3), H, the
            // record size and C
            put32(out, (uint32_t)n_cls[0] | ((uint32_t)n_cls[2] << 16));
            put32(out, (uint32_t)n_cls[1] | ((uint32_t)n_cls[3] << 16));
            put32(out, unsafe ? 0u : (uint32_t)np_halvings);
            put32(out, (uint32_t)rec_bytes);
            for (int k = 0; k < 4; ++k) put64(out, unsafe ? 0ull : (uint64_t)C[k]);
            // a fast term's layout as its reader takes it: part offsets in
            // 16-byte units, the first PhasePairs row, the NodePhases
            // valuation mod 4 and the constants' offset
            uint32_t lay[3] = {0u, 0u, 0u};
            if (!unsafe) {
                TermHdr lh = {};
                lh.n_np = (uint32_t)n_np; lh.n_hp = (uint32_t)n_hp; lh.n_pp = (uint32_t)n_pp; lh.n_ph = (uint32_t)n_ph;
                lh.flags = flags;
                lh.n_cls[0] = (uint32_t)n_cls[0]; lh.n_cls[1] = (uint32_t)n_cls[2];  // run order j = 0, 2, 1, 3
                lh.n_cls[2] = (uint32_t)n_cls[1]; lh.n_cls[3] = (uint32_t)n_cls[3];
                const int meta = layout_meta_off(lh), tab = layout_pair_tab_off(lh), step = layout_pair_step_off(lh);
                const int npl = layout_npl_off(lh), blk = layout_blocks_off(lh), row0 = ph_row0;
                if (blk != meta + (int)blocks_at || ((meta | tab | step | npl | blk) & 15) || blk >= (1 << 20) ||
                    row0 > 0xFFFF) {
                    err = gname + ": internal error: term layout";
                    return KSIM_ERR_UNSUPPORTED;
                }
                lay[0] = (uint32_t)(tab >> 4) | ((uint32_t)(step >> 4) << 16);
                lay[1] = (uint32_t)(npl >> 4) | ((uint32_t)(blk >> 4) << 16);
                lay[2] = (uint32_t)row0 | (layout_nu0(lh) << 16) | ((uint32_t)(meta >> 4) << 18);
            }
            put32(out, nb);
            for (uint32_t x : lay) put32(out, x);
            if (g.pf_has_approx) {
                double ar = g.pf_approx_f32[2 * (size_t)t], ai = g.pf_approx_f32[2 * (size_t)t + 1];
                uint64_t u;
                std::memcpy(&u, &ar, 8);
                put64(out, u);
                std::memcpy(&u, &ai, 8);
                put64(out, u);
            }
            out.insert(out.end(), body.begin(), body.end());
            (void)ff64;
            const int64_t tb = (int64_t)out.size() - start;
            img.max_term_bytes = std::max(img.max_term_bytes, tb);
            img.n_terms += 1;
            img.n_slow_terms += unsafe ? 1 : 0;
            img.n_narrow_terms += (flags & TF_NARROW) ? 1 : 0;
            img.n_hybrid_terms += (flags & TF_HYBRID) ? 1 : 0;
            img.n_columns += n_np + n_hp + n_pp + n_ph;
            img.work_ops += term_work(W, flags, n_cls, n_hp, n_pp, n_ph, (int)nb, (int)sum_iter);
        }
        toff.push_back((int64_t)out.size());
        img.work_ops += graph_work(W);
        gd.stream_bytes = (int64_t)out.size() - gd.stream_off;
        gd.n_chunks = 0;
        gd.first_chunk = 0;
    }
    std::memcpy(out.data(), img.gdir.data(), sizeof(GraphDir) * (size_t)n_graphs);
    return KSIM_OK;
}

bool make_chunks(const HostImage &img, int64_t slot_bytes, std::vector<ChunkDir> &out)
{
    out.clear();
    for (int k = 0; k < img.n_graphs; ++k) {
        const std::vector<int64_t> &to = img.term_off[k];
        const int G = (int)to.size() - 1;
        if (G <= 0) {
            ChunkDir c = {};
            c.off = img.gdir[k].stream_off;
            c.graph = k;
            c.end_of_graph = 1;
            out.push_back(c);
            continue;
        }
        int t = 0;
        while (t < G) {
            ChunkDir c = {};
            c.off = to[t];
            c.graph = k;
            int u = t;
            while (u < G && to[u + 1] - c.off <= slot_bytes) ++u;
            if (u == t) return false;  // a single term does not fit
            c.bytes = (int32_t)(to[u] - c.off);
            c.n_terms = u - t;
            c.end_of_graph = (u == G) ? 1 : 0;
            out.push_back(c);
            t = u;
        }
    }
    return true;
}

}  // namespace ksim
