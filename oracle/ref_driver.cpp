// ref_driver.cpp — drives the reference's own zx_eval.hpp on the CPU.
//
// TEST INFRASTRUCTURE ONLY (the "reference" CPU baseline and a parity pin for
// oracle/ksim_oracle.c).  oracle/Makefile compiles this file against the
// reference's src/cpp/ksim/zx_eval.hpp where it lies in the reference tree
// (unmodified) and oracle/kokkos_shim/Kokkos_Core.hpp, into oracle/_ref/.
//
// What is restated here (kokkos_sim.cpp itself needs Kokkos + nanobind, which
// are absent):
//   - packing of the per-graph arrays into meta / u8 / i32 / apx buffers with
//     int32 offsets, in the reference's field order   kokkos_sim.cpp:91-149
//   - the per-shot sample loop                          kokkos_sim.cpp:214-230
//   - seed mixing and the xorshift64 uniform           kokkos_sim.cpp:43-46,215-217
//   - eval_abs's "all params through the f view"        kokkos_sim.cpp:157-185
// eval_graph, zw_mul, zw_reduce and zw_unit are the reference's own code.
// Built with -ffp-contract=off -fwrapv (int64 wraps as on the GPU).
#include <Kokkos_Core.hpp>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "zx_eval.hpp"

#include "../include/ksim_b200.h"

extern "C" double oracle_philox_uniform_ref(uint64_t seed, uint64_t shot, uint32_t output);

namespace {

struct HostComponent {
    std::vector<int32_t> meta;
    std::vector<uint8_t> u8;
    std::vector<int32_t> i32;
    std::vector<double> apx;
    DevComponent dev;
};

// Append one array, returning its element offset (int32 as in the reference).
template <class T> int32_t push(std::vector<T> &buf, const T *p, size_t n)
{
    int32_t off = (int32_t)buf.size();
    if (n) buf.insert(buf.end(), p, p + n);
    return off;
}

void build(const ksim_graph_desc *gs, int n_graphs, int F, HostComponent &hc)
{
    for (int k = 0; k < n_graphs; ++k) {
        const ksim_graph_desc &g = gs[k];
        const size_t G = (size_t)g.G, P = (size_t)g.P;
        int32_t m[NMETA] = {};
        m[M_G] = g.G; m[M_P] = g.P;
        m[M_TNP] = g.Tnp; m[M_THP] = g.Thp; m[M_TPP] = g.Tpp; m[M_TPH] = g.Tph;
        m[M_NP_PH] = push(hc.u8, g.np_phases, G * g.Tnp);
        m[M_NP_PAR] = push(hc.u8, g.np_params, G * g.Tnp * P);
        m[M_NP_CNT] = push(hc.i32, g.np_counts, G);
        m[M_HP_CO] = push(hc.u8, g.hp_coeffs, G * g.Thp);
        m[M_HP_PAR] = push(hc.u8, g.hp_params, G * g.Thp * P);
        m[M_PP_PSC] = push(hc.u8, g.pp_psi_c, G * g.Tpp);
        m[M_PP_PSP] = push(hc.u8, g.pp_psi_p, G * g.Tpp * P);
        m[M_PP_PHC] = push(hc.u8, g.pp_phi_c, G * g.Tpp);
        m[M_PP_PHP] = push(hc.u8, g.pp_phi_p, G * g.Tpp * P);
        m[M_PH_AL] = push(hc.u8, g.ph_alpha, G * g.Tph);
        m[M_PH_ALP] = push(hc.u8, g.ph_alpha_p, G * g.Tph * P);
        m[M_PH_BE] = push(hc.u8, g.ph_beta, G * g.Tph);
        m[M_PH_BEP] = push(hc.u8, g.ph_beta_p, G * g.Tph * P);
        m[M_PH_CNT] = push(hc.i32, g.ph_counts, G);
        m[M_PF_IDX] = push(hc.u8, g.pf_phase_idx, G);
        m[M_PF_FF] = push(hc.i32, g.pf_floatfactor, G * 4);
        m[M_PF_P2] = push(hc.i32, g.pf_power2, G);
        m[M_PF_APX] = (int32_t)hc.apx.size();
        for (size_t i = 0; i < 2 * G; ++i)
            hc.apx.push_back(g.pf_approx_f32 ? (double)g.pf_approx_f32[i] : 0.0);
        m[M_HAS_APX] = g.pf_has_approx ? 1 : 0;
        hc.meta.insert(hc.meta.end(), m, m + NMETA);
    }
    if (hc.u8.empty()) hc.u8.push_back(0);
    if (hc.i32.empty()) hc.i32.push_back(0);
    if (hc.apx.empty()) hc.apx.push_back(0.0);
    hc.dev.n_out = n_graphs - 1;
    hc.dev.F = F;
    hc.dev.n_graphs = n_graphs;
    hc.dev.meta = Kokkos::View<const int32_t *, DeviceSpace>(hc.meta.data(), hc.meta.size());
    hc.dev.u8 = Kokkos::View<const uint8_t *, DeviceSpace>(hc.u8.data(), hc.u8.size());
    hc.dev.i32 = Kokkos::View<const int32_t *, DeviceSpace>(hc.i32.data(), hc.i32.size());
    hc.dev.apx = Kokkos::View<const double *, DeviceSpace>(hc.apx.data(), hc.apx.size());
}

// 2-D row-major byte view, the shape eval_graph reads f and m through.
struct Rows {
    const uint8_t *p;
    size_t stride;
    int operator()(size_t s, size_t j) const { return p[s * stride + j]; }
};

double xorshift_uniform(uint64_t &s)
{
    s ^= s << 13; s ^= s >> 7; s ^= s << 17;
    return (double)(s >> 11) * (1.0 / (double)(1ULL << 53));
}

}  // namespace

extern "C" int oracle_ref_sample(const ksim_graph_desc *graphs, int n_graphs, int F,
                                 const uint8_t *f_sel, int64_t B, int64_t shot_offset,
                                 uint64_t seed, int rng_mode, uint8_t *out, double *amp,
                                 int n_threads)
{
    if (n_graphs < 1 || F < 0 || B < 0) return 1;
    HostComponent hc;
    build(graphs, n_graphs, F, hc);
    const int n_out = n_graphs - 1;
    const size_t ncol = (size_t)std::max(n_out, 1);
    std::memset(out, 0, (size_t)B * ncol);
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#else
    (void)n_threads;
#endif
    const DevComponent C = hc.dev;
    Rows f{f_sel, (size_t)F};
    Rows m{out, ncol};
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t si = 0; si < B; ++si) {
        const int s = (int)si;  // eval_graph indexes shots with int, as kokkos_sim does
        const uint64_t gs = (uint64_t)(shot_offset + si);
        uint64_t rng = seed ^ (gs * 0x9e3779b97f4a7c15ULL);
        rng ^= rng >> 30; rng *= 0xbf58476d1ce4e5b9ULL;
        rng ^= rng >> 27; rng = rng ? rng : 1ULL;
        double re, im;
        eval_graph(C, 0, s, 0, 0, f, m, re, im);
        double prev = std::sqrt(re * re + im * im);
        if (amp) amp[(size_t)si * (size_t)(n_out + 1)] = prev;
        for (int i = 0; i < n_out; ++i) {
            eval_graph(C, i + 1, s, i, 1, f, m, re, im);
            double p1 = std::sqrt(re * re + im * im);
            if (amp) amp[(size_t)si * (size_t)(n_out + 1) + 1 + i] = p1;
            double u = rng_mode == KSIM_RNG_PHILOX ? oracle_philox_uniform_ref(seed, gs, (uint32_t)i)
                                                   : xorshift_uniform(rng);
            int bit = u < (p1 / prev) ? 1 : 0;
            out[(size_t)si * ncol + i] = (uint8_t)bit;
            prev = bit ? p1 : (prev - p1);
        }
    }
    return 0;
}

extern "C" int oracle_ref_eval(const ksim_graph_desc *graphs, int n_graphs, int gi,
                               const uint8_t *params, int64_t B, int64_t P, double *out_re_im)
{
    if (gi < 0 || gi >= n_graphs || B < 0 || P < 0) return 1;
    HostComponent hc;
    build(graphs, n_graphs, (int)P, hc);
    DevComponent C = hc.dev;
    C.F = (int)P;  // every parameter comes through the f view
    Rows f{params, (size_t)P};
#pragma omp parallel for schedule(static)
    for (int64_t si = 0; si < B; ++si) {
        double re, im;
        eval_graph(C, gi, (int)si, 0, 0, f, f, re, im);
        out_re_im[2 * si] = re;
        out_re_im[2 * si + 1] = im;
    }
    return 0;
}

// Philox4x32-10 (Salmon et al., SC'11) for the counter-based uniform mode.
extern "C" double oracle_philox_uniform_ref(uint64_t seed, uint64_t shot, uint32_t output)
{
    uint32_t c0 = (uint32_t)shot, c1 = (uint32_t)(shot >> 32), c2 = output, c3 = 0;
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c0 = n0; c1 = (uint32_t)p1; c2 = n2; c3 = (uint32_t)p0;
    }
    uint64_t bits = ((uint64_t)c1 << 32) | c0;
    return (double)(bits >> 11) * (1.0 / 9007199254740992.0);
}

extern "C" int oracle_ref_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
