"""GPU parity: the sm_100a kernels against the oracle, through the C ABI.

Bit-exact targets (the reference kernel's semantics, zx_eval.hpp +
kokkos_sim.cpp:214-230): every per-term numerator (a, b, c, d, pw), every
amplitude double, every |A_k| and every sampled bit, for both uniform streams.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import pytest

from helpers import golden_names, load_golden, same_bits
from ksim_b200 import synth
from ksim_b200.program import FlatComponent

pytestmark = pytest.mark.gpu


def _component(graphs, F):
    from ksim_b200.kokkos_sim import Component
    return Component(graphs, F)


def device_sample(comp, f, seed, mode, shot_offset=0):
    """Sample through ksim_component_sample_device with torch-owned buffers;
    returns (bits (B, n_out), amp (B, n_out+1))."""
    import torch
    from ksim_b200 import _abi
    B = f.shape[0]
    n_out = comp.n_out
    d_f = torch.from_numpy(np.ascontiguousarray(f, np.uint8).copy()).cuda()
    d_out = torch.zeros((B, max(n_out, 1)), dtype=torch.uint8, device="cuda")
    d_amp = torch.zeros((B, n_out + 1), dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    _abi.check(_abi.lib().ksim_component_sample_device(
        comp.handle, ctypes.c_void_p(d_f.data_ptr()), B, shot_offset, seed, mode,
        ctypes.c_void_p(d_out.data_ptr()), max(n_out, 1), 0, ctypes.c_void_p(d_amp.data_ptr()),
        ctypes.c_void_p(st)))
    torch.cuda.synchronize()
    return d_out.cpu().numpy()[:, :n_out], d_amp.cpu().numpy()


def _random_component(seed):
    rng = np.random.default_rng(seed)
    comp = synth.random_component(rng, n_out=int(rng.integers(1, 12)), F=int(rng.integers(0, 150)),
                                  t=int(rng.integers(1, 18)), f_prob=0.05)
    return rng, comp, int(np.asarray(comp.f_selection).shape[0])


@pytest.mark.parametrize("name", golden_names())
def test_golden_fixtures(cuda_device, name):
    prog, d = load_golden(name)
    for ci, comp in enumerate(prog.components):
        F = int(np.asarray(comp.f_selection).shape[0])
        kc = _component(comp.graphs, F)
        for gi in range(len(comp.graphs)):
            pv = d[f"c{ci}_g{gi}_params"]
            assert same_bits(kc.eval(gi, pv), d[f"c{ci}_g{gi}_ref_amp"]), (name, gi)
        for seed in (11, 2**63 + 12345):
            for mode in (0, 1):
                bits = kc.sample(d[f"c{ci}_f"], seed, rng_mode=mode)
                assert np.array_equal(bits, d[f"c{ci}_bits_s{seed % 1000}_m{mode}"]), (name, seed, mode)
                b2, amp = device_sample(kc, d[f"c{ci}_f"], seed, mode)
                assert same_bits(amp, d[f"c{ci}_amp_s{seed % 1000}_m{mode}"]), (name, seed, mode)


@pytest.mark.parametrize("seed", range(8))
def test_eval_and_terms_match_oracle(cuda_device, oracle_port, seed):
    rng, comp, F = _random_component(seed)
    kc = _component(comp.graphs, F)
    po = oracle_port.PortOracle(comp.graphs, F)
    for gi, g in enumerate(comp.graphs):
        P = g.np_params.shape[2]
        pv = rng.integers(0, 2, size=(257, P)).astype(np.uint8)
        assert np.array_equal(kc.eval_terms(gi, pv), po.eval_terms(gi, pv)), gi
        assert same_bits(kc.eval(gi, pv), po.eval(gi, pv)), gi
        assert same_bits(kc.eval_abs(gi, pv), po.eval_abs(gi, pv)), gi


@pytest.mark.parametrize("seed", range(8))
def test_sample_matches_oracle(cuda_device, oracle_port, seed):
    rng, comp, F = _random_component(100 + seed)
    kc = _component(comp.graphs, F)
    po = oracle_port.PortOracle(comp.graphs, F)
    f = synth.sample_f(rng, 3000, F, 0.05)
    for mode in (0, 1):
        want, want_amp = po.sample(f, 1000 + seed, mode, return_amp=True)
        assert np.array_equal(kc.sample(f, 1000 + seed, rng_mode=mode), want)
        bits, amp = device_sample(kc, f, 1000 + seed, mode)
        assert np.array_equal(bits, want[:, :kc.n_out]) and same_bits(amp, want_amp)


def test_launch_shapes_agree(cuda_device, oracle_port):
    rng, comp, F = _random_component(7)
    kc = _component(comp.graphs, F)
    f = synth.sample_f(rng, 5000, F, 0.05)
    want = oracle_port.PortOracle(comp.graphs, F).sample(f, 77, 0)
    mtb = kc.stats()["max_term_bytes"]
    for threads in (32, 64, 128, 256):
        for staged in (0, 1):
            for slot in sorted({(mtb + 15) // 16 * 16, 16384, 65536}):
                kc.set_launch(threads=threads, staged=staged, slot_bytes=slot)
                assert np.array_equal(kc.sample(f, 77), want), (threads, staged, slot)


def test_exact_path_and_wrap_on_gpu(cuda_device, oracle_port):
    from ksim_b200._abi import FLAG_INT64_RISK
    rng = np.random.default_rng(250)
    gs = [synth.random_graph(rng, 3, 20 + k, 250, 3, 3, 40) for k in range(4)]
    for g in gs:
        # 250 factors (1 + w^(1+4 par)): |coefficients| grow ~5.8^(n/4) and wrap int64
        g.np_phases[:] = 1
        g.np_params[:] = 0
        g.np_params[:, ::7, 0] = 1
        g.np_counts[:] = 250
    comp = FlatComponent((0, 1, 2), np.arange(20, dtype=np.int32), gs)
    kc = _component(comp.graphs, 20)
    po = oracle_port.PortOracle(comp.graphs, 20)
    assert kc.stats()["slow_terms"] == kc.stats()["terms"]
    for gi, g in enumerate(gs):
        pv = rng.integers(0, 2, size=(64, g.np_params.shape[2])).astype(np.uint8)
        assert np.array_equal(kc.eval_terms(gi, pv), po.eval_terms(gi, pv))
        assert same_bits(kc.eval(gi, pv), po.eval(gi, pv))
    f = synth.sample_f(rng, 256, 20, 0.1)
    assert np.array_equal(kc.sample(f, 3), po.sample(f, 3, 0))
    assert kc.status() & FLAG_INT64_RISK


def test_edge_cases_gpu(cuda_device, oracle_port):
    rng = np.random.default_rng(77)
    comp = synth.random_component(rng, n_out=4, F=5, t=6, calibrate=False)
    for g in comp.graphs:
        G = g.pf_phase_idx.shape[0]
        g.pf_approx = (rng.normal(size=G) + 1j * rng.normal(size=G)).astype(np.complex64)
        g.pf_has_approx = True
        g.np_counts[0] = -3
        g.np_phases[:] = g.np_phases + 8 * rng.integers(0, 3, size=g.np_phases.shape)
        g.pf_phase_idx[:] = g.pf_phase_idx + 8
    comp.graphs[2].pf_phase_idx = comp.graphs[2].pf_phase_idx[:0]
    for name in ("np_phases", "hp_coeffs", "pp_psi_c", "pp_phi_c", "ph_alpha", "ph_beta",
                 "np_params", "hp_params", "pp_psi_p", "pp_phi_p", "ph_alpha_p", "ph_beta_p",
                 "np_counts", "ph_counts", "pf_power2", "pf_approx", "pf_floatfactor"):
        setattr(comp.graphs[2], name, getattr(comp.graphs[2], name)[:0])
    kc = _component(comp.graphs, 5)
    po = oracle_port.PortOracle(comp.graphs, 5)
    f = synth.sample_f(rng, 1000, 5, 0.2)
    for mode in (0, 1):
        want, wamp = po.sample(f, 5, mode, return_amp=True)
        bits, amp = device_sample(kc, f, 5, mode)
        assert np.array_equal(bits, want[:, :4]) and same_bits(amp, wamp)


@pytest.mark.parametrize("base", [-1060, -1022, -1005, 960, 1005])
def test_scales_near_and_beyond_the_normal_range(cuda_device, oracle_port, base):
    """power2 shifted by `base`: terms whose scales 2^(pw + power2) can reach
    subnormal or infinite values take the general scale (pow2i), the others
    the exponent-bits one (TF_EXP).  Per-term numerators, amplitudes and
    sampled bits must be the oracle's on both sides of the boundary (at these
    scales |A|^2 under- or overflows, so the bits degenerate as in the
    reference; the shifts stop short of sums of opposite infinities, whose
    NaN bit patterns differ between host and device)."""
    rng = np.random.default_rng(1300 + abs(base))
    comp = synth.random_component(rng, n_out=6, F=20, t=10, f_prob=0.1)
    for g in comp.graphs:
        g.pf_power2 = (g.pf_power2.astype(np.int64) + base).astype(np.int32)
    kc = _component(comp.graphs, 20)
    po = oracle_port.PortOracle(comp.graphs, 20)
    for gi, g in enumerate(comp.graphs):
        pv = rng.integers(0, 2, size=(128, g.np_params.shape[2])).astype(np.uint8)
        assert np.array_equal(kc.eval_terms(gi, pv), po.eval_terms(gi, pv))
        assert same_bits(kc.eval(gi, pv), po.eval(gi, pv))
    f = synth.sample_f(rng, 3000, 20, 0.1)
    for mode in (0, 1):
        want, wamp = po.sample(f, 11, mode, return_amp=True)
        bits, amp = device_sample(kc, f, 11, mode)
        assert np.array_equal(bits, want[:, :6]) and same_bits(amp, wamp)


def test_reference_api_edges(cuda_device):
    prog, _ = synth.htkh(1)
    graphs = prog.components[0].graphs
    kc = _component(graphs, 0)
    assert kc.n_out == 1
    assert kc.sample(np.zeros((0, 0), np.uint8), 1).shape == (0, 1)
    with pytest.raises(ValueError):
        kc.sample(np.zeros((4, 3), np.uint8), 1)     # kokkos_sim.cpp:193-194
    with pytest.raises(TypeError):
        kc.sample(np.zeros((4, 0), np.uint8), -1)    # not a uint64
    with pytest.raises(TypeError):
        kc.sample(np.zeros((4, 0), np.uint8), 2**64)
    # n_out = 0: one zero column, as the reference pads to max(n_out, 1)
    k0 = _component(graphs[:1], 0)
    out = k0.sample(np.zeros((5, 0), np.uint8), 3)
    assert out.shape == (5, 1) and not out.any()


def test_program_sample_matches_oracle(cuda_device, oracle_port):
    from ksim_b200.sampler import B200ProgramSampler
    rng = np.random.default_rng(31)
    prog, nf = synth.multi_component_program(rng, [(3, 5, 3), (6, 12, 6), (2, 0, 2), (5, 40, 8)])
    f = synth.sample_f(rng, 4000, nf, 0.05)
    s = B200ProgramSampler(prog)
    for mode in (0, 1):
        want = oracle_port.program_sample(prog, f, 2024, rng_mode=mode)
        got = s.sample(f, 2024, rng_mode=mode)
        assert got.shape == (4000, prog.num_outputs)
        assert np.array_equal(got, want)
    # extra f columns beyond those selected are allowed
    wide = np.concatenate([f, np.ones((4000, 5), np.uint8)], axis=1)
    assert np.array_equal(s.sample(wide, 2024), oracle_port.program_sample(prog, wide, 2024))


def test_shot_offset_split_invariance(cuda_device):
    rng, comp, F = _random_component(55)
    kc = _component(comp.graphs, F)
    f = synth.sample_f(rng, 9000, F, 0.05)
    for mode in (0, 1):
        whole, wamp = device_sample(kc, f, 9, mode)
        a, aa = device_sample(kc, f[:4000], 9, mode, shot_offset=0)
        b, ba = device_sample(kc, f[4000:], 9, mode, shot_offset=4000)
        assert np.array_equal(whole, np.concatenate([a, b]))
        assert same_bits(wamp, np.concatenate([aa, ba]))


@pytest.mark.parametrize("k", [1, 2, 3])
def test_htkh_p1(cuda_device, k):
    """tests/test_nonclifford.py:105-121: P(1) within 5 sigma of sin^2(k pi/8)."""
    from ksim_b200.sampler import B200ProgramSampler
    prog, exact = synth.htkh(k)
    n = 20_000
    p1 = B200ProgramSampler(prog).sample(np.zeros((n, 0), np.uint8), seed=11)[:, 0].mean()
    assert abs(p1 - exact) < 5 * math.sqrt(exact * (1 - exact) / n)


def test_t_depth_two_p1(cuda_device):
    """tests/test_nonclifford.py:184-194: H T H T H gives 1/4."""
    from ksim_b200.sampler import B200ProgramSampler
    prog, exact = synth.t_depth_two()
    n = 20_000
    p1 = B200ProgramSampler(prog).sample(np.zeros((n, 0), np.uint8), seed=11)[:, 0].mean()
    assert abs(p1 - exact) < 5 * math.sqrt(exact * (1 - exact) / n)


def test_mixture_distribution(cuda_device):
    from ksim_b200.sampler import B200ProgramSampler
    rng = np.random.default_rng(22)
    prog, F, prob = synth.mixture(rng, n_out=4, r=3, F=2)
    n = 200_000
    f = synth.sample_f(rng, n, F, 0.3)
    bits = B200ProgramSampler(prog).sample(f, 5, rng_mode=1)
    for fv in ((0, 0), (1, 0), (0, 1), (1, 1)):
        rows = (f[:, 0] == fv[0]) & (f[:, 1] == fv[1])
        codes = bits[rows] @ (1 << np.arange(4))
        counts = np.bincount(codes, minlength=16)
        m = int(rows.sum())
        for c in range(16):
            p = prob(list(fv), [(c >> j) & 1 for j in range(4)])
            assert abs(counts[c] / m - p) < 5 * math.sqrt(max(p * (1 - p), 1e-12) / m) + 1e-9


@pytest.mark.parametrize("Tnp,Tph", [(40, 30), (60, 10)])
def test_hybrid_and_wide_terms_on_gpu(cuda_device, oracle_port, Tnp, Tph):
    """Terms whose NodePhases block fits 32-bit words but whose PhasePairs do
    not (hybrid path), next to 32-bit and 64-bit terms: numerators, amplitudes
    and bits equal the oracle's."""
    rng = np.random.default_rng(7000 + Tnp)
    gs = [synth.random_graph(rng, 6, 20 + k, Tnp, 3, 3, Tph) for k in range(4)]
    comp = FlatComponent((0, 1, 2), np.arange(20, dtype=np.int32), gs)
    kc = _component(comp.graphs, 20)
    po = oracle_port.PortOracle(comp.graphs, 20)
    for gi, g in enumerate(comp.graphs):
        pv = rng.integers(0, 2, size=(129, g.np_params.shape[2])).astype(np.uint8)
        assert np.array_equal(kc.eval_terms(gi, pv), po.eval_terms(gi, pv)), gi
        assert same_bits(kc.eval(gi, pv), po.eval(gi, pv)), gi
    f = synth.sample_f(rng, 2000, 20, 0.1)
    for mode in (0, 1):
        want, want_amp = po.sample(f, 99, mode, return_amp=True)
        bits, amp = device_sample(kc, f, 99, mode)
        assert np.array_equal(bits, want[:, :kc.n_out]) and same_bits(amp, want_amp)


@pytest.mark.parametrize("Tnp,Tph,seed,kind", [(40, 12, 2, "narrow"), (50, 16, 5, "narrow+hybrid"),
                                                (60, 10, 4, "all")])
def test_kernel_per_term_path_set(cuda_device, oracle_port, Tnp, Tph, seed, kind):
    """The plain sampler runs a kernel compiled for the term paths a component
    uses (every term on 32-bit words; 32-bit and hybrid; any): each equals the
    oracle, bits and |A_k|, for both uniform streams and for a shot offset."""
    from ksim_b200.perfmodel import component_work
    rng = np.random.default_rng(seed)
    gs = [synth.random_graph(rng, 6, 20 + k, Tnp, 3, 3, Tph) for k in range(4)]
    comp = FlatComponent((0, 1, 2), np.arange(20, dtype=np.int32), gs)
    w = component_work(comp)
    got_kind = ("narrow" if w["hybrid_terms"] + w["wide_terms"] + w["exact_terms"] == 0 else
                "narrow+hybrid" if w["wide_terms"] + w["exact_terms"] == 0 else "all")
    assert got_kind == kind, w
    kc = _component(comp.graphs, 20)
    po = oracle_port.PortOracle(comp.graphs, 20)
    f = synth.sample_f(rng, 3000, 20, 0.1)
    for mode, off in ((0, 0), (1, 0), (1, 777)):
        want, want_amp = po.sample(f, 123, mode, return_amp=True, shot_offset=off)
        bits, amp = device_sample(kc, f, 123, mode, shot_offset=off)
        assert np.array_equal(bits, want[:, :kc.n_out]) and same_bits(amp, want_amp), (mode, off)
