"""The device evaluator, compiled for the CPU, against the oracle.

ksim_b200/csrc/zring.cuh replaces the reference's 16-multiply products and
explicit evenness tests by signed rotations and a host-precomputed
valuation schedule (see its header).  These tests run that exact code (built
with g++ from the same header, over the same packed image) against the C
restatement of zx_eval.hpp: every per-term numerator (a, b, c, d, pw), every
amplitude and every sampled bit must be identical.
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import HostEmu, golden_names, load_golden, same_bits
from ksim_b200 import synth
from ksim_b200.program import FlatComponent


def _check_component(hostemu, oracle_port, comp, F, rng, B=128):
    he = HostEmu(hostemu, comp.graphs, F)
    po = oracle_port.PortOracle(comp.graphs, F)
    for gi, g in enumerate(comp.graphs):
        P = g.np_params.shape[2]
        pv = rng.integers(0, 2, size=(24, P)).astype(np.uint8)
        assert np.array_equal(he.eval_terms(gi, pv), po.eval_terms(gi, pv)), gi
        assert same_bits(he.eval(gi, pv), po.eval(gi, pv)), gi
    f = synth.sample_f(rng, B, F, 0.05)
    for mode in (0, 1):
        bits, amp = he.sample(f, 4242, mode)
        rb, ra = po.sample(f, 4242, mode, return_amp=True)
        assert np.array_equal(bits, rb) and same_bits(amp, ra), mode
    return he.stats()


@pytest.mark.parametrize("base", [-1060, -1022, -1005, 960, 1005])
def test_scales_near_and_beyond_the_normal_range(hostemu, oracle_port, base):
    """power2 shifted by `base`: terms whose scales 2^(pw + power2) can be
    subnormal or infinite take pow2i, the others the exponent-bits scale
    (TF_EXP); both must give the oracle's doubles (shifts short of sums of
    opposite infinities, whose NaN bit patterns need not agree)."""
    rng = np.random.default_rng(2600 + abs(base))
    comp = synth.random_component(rng, n_out=5, F=16, t=9, f_prob=0.1)
    for g in comp.graphs:
        g.pf_power2 = (g.pf_power2.astype(np.int64) + base).astype(np.int32)
    _check_component(hostemu, oracle_port, comp, 16, rng)


@pytest.mark.parametrize("seed", range(10))
def test_random_components(hostemu, oracle_port, seed):
    rng = np.random.default_rng(seed)
    comp = synth.random_component(rng, n_out=int(rng.integers(1, 10)), F=int(rng.integers(0, 140)),
                                  t=int(rng.integers(1, 20)), f_prob=0.05)
    _check_component(hostemu, oracle_port, comp, int(np.asarray(comp.f_selection).shape[0]), rng)


@pytest.mark.parametrize("Tnp,Tph", [(24, 4), (40, 30), (60, 10), (130, 20), (250, 40)])
def test_long_terms_exact_path(hostemu, oracle_port, Tnp, Tph):
    """Short terms run on 32-bit words, longer ones on 64-bit words, and terms
    the host cannot prove overflow-free take the exact path."""
    rng = np.random.default_rng(Tnp)
    gs = [synth.random_graph(rng, 4, 20 + k, Tnp, 3, 3, Tph) for k in range(4)]
    comp = FlatComponent((0, 1, 2), np.arange(20, dtype=np.int32), gs)
    st = _check_component(hostemu, oracle_port, comp, 20, rng, B=32)
    wide = st["terms"] - st["slow_terms"] - st["narrow_terms"] - st["hybrid_terms"]
    if Tnp == 24:
        assert st["narrow_terms"] == st["terms"]
    if Tnp == 60:
        assert wide + st["hybrid_terms"] > 0
    if Tnp >= 250:
        assert st["slow_terms"] == st["terms"]


@pytest.mark.parametrize("Tnp,Tph", [(24, 4), (40, 30), (60, 10), (250, 40)])
def test_two_shots_per_thread_path(hostemu, oracle_port, Tnp, Tph):
    """Evaluating two parameter rows at once (the kernels' two-shots-per-thread
    path, on the 32-bit, 64-bit and exact term paths) gives the same
    numerators and amplitudes as one row at a time, for even and odd counts."""
    rng = np.random.default_rng(1000 + Tnp)
    gs = [synth.random_graph(rng, 5, 20 + k, Tnp, 3, 3, Tph) for k in range(3)]
    he = HostEmu(hostemu, gs, 20)
    po = oracle_port.PortOracle(gs, 20)
    for gi, g in enumerate(gs):
        P = g.np_params.shape[2]
        for B in (1, 2, 7, 16):
            pv = rng.integers(0, 2, size=(B, P)).astype(np.uint8)
            want = po.eval_terms(gi, pv)
            assert np.array_equal(he.eval_terms(gi, pv, pairs=True), want), (gi, B)
            assert same_bits(he.eval(gi, pv, pairs=True), he.eval(gi, pv)), (gi, B)


def test_every_term_path_is_taken(hostemu):
    """The parametrised components above cover the 32-bit, 64-bit and exact paths."""
    counts = {"narrow": 0, "hybrid": 0, "wide": 0, "slow": 0}
    for Tnp, Tph in [(24, 4), (40, 30), (60, 10), (130, 20), (250, 40)]:
        rng = np.random.default_rng(Tnp)
        gs = [synth.random_graph(rng, 4, 20 + k, Tnp, 3, 3, Tph) for k in range(4)]
        st = HostEmu(hostemu, gs, 20).stats()
        counts["narrow"] += st["narrow_terms"]
        counts["hybrid"] += st["hybrid_terms"]
        counts["slow"] += st["slow_terms"]
        counts["wide"] += st["terms"] - st["narrow_terms"] - st["slow_terms"] - st["hybrid_terms"]
    assert all(v > 0 for v in counts.values()), counts


def test_int64_wrap_is_reproduced_and_flagged(hostemu, oracle_port):
    """A term of 250 (1 + w^(1+4 par)) factors overflows int64; the exact path
    wraps exactly like the reference and raises the risk flag."""
    import ctypes
    rng = np.random.default_rng(250)
    gs = [synth.random_graph(rng, 3, 20 + k, 250, 3, 3, 40) for k in range(4)]
    for g in gs:
        g.np_phases[:] = 1
        g.np_params[:] = 0
        g.np_params[:, ::7, 0] = 1
        g.np_counts[:] = 250
    comp = FlatComponent((0, 1, 2), np.arange(20, dtype=np.int32), gs)
    _check_component(hostemu, oracle_port, comp, 20, rng, B=16)
    he = HostEmu(hostemu, comp.graphs, 20)
    pv = rng.integers(0, 2, size=(8, 21)).astype(np.uint8)
    out = np.zeros((8, 2))
    risk = ctypes.c_uint32(0)
    assert hostemu.hostemu_eval(he.descs, 4, 20, 1, pv.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                                8, 21, 0, out.ctypes.data, ctypes.addressof(risk)) == 0
    assert risk.value == 1
    assert np.abs(he.eval_terms(1, pv)[..., :4].astype(float)).max() > 2.0**62


def test_edge_cases(hostemu, oracle_port):
    rng = np.random.default_rng(77)
    comp = synth.random_component(rng, n_out=4, F=5, t=6, calibrate=False)
    for g in comp.graphs:
        G = g.pf_phase_idx.shape[0]
        g.pf_approx = (rng.normal(size=G) + 1j * rng.normal(size=G)).astype(np.complex64)
        g.pf_has_approx = True
        g.np_counts[0] = -3                      # an empty loop in the reference
        g.np_phases[:] = g.np_phases + 8 * rng.integers(0, 3, size=g.np_phases.shape)
        g.hp_coeffs[:] = np.where(g.hp_coeffs > 0, g.hp_coeffs + 8, 0)
        g.pp_psi_c[:] = g.pp_psi_c + 2 * rng.integers(0, 2, size=g.pp_psi_c.shape)
        g.pf_phase_idx[:] = g.pf_phase_idx + 8
    _check_component(hostemu, oracle_port, comp, 5, rng)


def test_params_beyond_f_plus_k(hostemu, oracle_port):
    """A graph with P > F + nm + 1 sees the trying bit on every extra position."""
    rng = np.random.default_rng(8)
    comp = synth.random_component(rng, n_out=3, F=4, t=5, calibrate=False)
    for g in comp.graphs:
        for name in ("np_params", "hp_params", "pp_psi_p", "pp_phi_p", "ph_alpha_p", "ph_beta_p"):
            a = getattr(g, name)
            extra = rng.integers(0, 2, size=a.shape[:2] + (3,)).astype(np.uint8)
            setattr(g, name, np.concatenate([a, extra], axis=2))
    _check_component(hostemu, oracle_port, comp, 4, rng)


def test_empty_graph(hostemu, oracle_port):
    rng = np.random.default_rng(9)
    comp = synth.random_component(rng, n_out=3, F=4, t=5, calibrate=False)
    g = comp.graphs[2]
    for name in ("np_phases", "hp_coeffs", "pp_psi_c", "pp_phi_c", "ph_alpha", "ph_beta",
                 "np_params", "hp_params", "pp_psi_p", "pp_phi_p", "ph_alpha_p", "ph_beta_p",
                 "np_counts", "ph_counts", "pf_phase_idx", "pf_power2", "pf_approx",
                 "pf_floatfactor"):
        setattr(g, name, getattr(g, name)[:0])
    _check_component(hostemu, oracle_port, comp, 4, rng)


@pytest.mark.parametrize("name", golden_names())
def test_golden_fixtures(hostemu, name):
    """The device evaluator reproduces the reference zx_eval.hpp fixtures."""
    prog, d = load_golden(name)
    for ci, comp in enumerate(prog.components):
        F = int(np.asarray(comp.f_selection).shape[0])
        he = HostEmu(hostemu, comp.graphs, F)
        for gi in range(len(comp.graphs)):
            assert same_bits(he.eval(gi, d[f"c{ci}_g{gi}_params"]), d[f"c{ci}_g{gi}_ref_amp"])
        for seed in (11, 2**63 + 12345):
            for mode in (0, 1):
                bits, amp = he.sample(d[f"c{ci}_f"], seed, mode)
                assert np.array_equal(bits, d[f"c{ci}_bits_s{seed % 1000}_m{mode}"])
                assert same_bits(amp, d[f"c{ci}_amp_s{seed % 1000}_m{mode}"])


def test_valuation_matches_evenness(hostemu):
    """nu(z) >= 4  <=>  all four coefficients even (z != 0): the identity the
    kernels' renormalisation schedule rests on."""
    rng = np.random.default_rng(3)
    for _ in range(4000):
        z = rng.integers(-40, 41, size=4).astype(np.int64)
        if not z.any():
            continue
        nu = hostemu.hostemu_valuation(z.ctypes.data)
        assert (nu >= 4) == bool(np.all(z % 2 == 0))
    # nu(1 - w) = 1, nu(1 + i) = 2, nu(2) = 4, nu(0) = 15 (the zero marker)
    for z, want in (([1, -1, 0, 0], 1), ([1, 0, 1, 0], 2), ([2, 0, 0, 0], 4), ([0, 0, 0, 0], 15)):
        assert hostemu.hostemu_valuation(np.array(z, np.int64).ctypes.data) == want


@pytest.mark.parametrize("Tnp", [1, 7, 33, 90])
def test_nodephases_by_sign_counts(hostemu, oracle_port, Tnp):
    """NodePhases blocks alone, on every path: the counted form (one constant
    times lambda^(m3 - m1), rotation w^(6 M), class-0 kill with the
    reference's pw) gives the reference's per-term numerators, dead terms
    included."""
    rng = np.random.default_rng(77 + Tnp)
    gs = [synth.random_graph(rng, 16, 12 + k, Tnp, 0, 0, 0, density=0.3) for k in range(3)]
    he = HostEmu(hostemu, gs, 12)
    po = oracle_port.PortOracle(gs, 12)
    dead = 0
    for gi, g in enumerate(gs):
        P = g.np_params.shape[2]
        pv = rng.integers(0, 2, size=(64, P)).astype(np.uint8)
        want = po.eval_terms(gi, pv)
        assert np.array_equal(he.eval_terms(gi, pv), want), gi
        assert np.array_equal(he.eval_terms(gi, pv, pairs=True), want), gi
        dead += int(((want[..., :4] == 0).all(-1) & (want[..., 4] > 0)).sum())
    if Tnp >= 7:
        assert dead > 0


@pytest.mark.parametrize("zero", ["alpha", "beta", "both"])
def test_phasepairs_with_a_zero_rotation(hostemu, oracle_port, zero):
    """PhasePairs columns with rotation class 0 on one side (1 + a + b - ab is
    2 or 2b: a select and one halving) give the reference's numerators,
    on every term path and for terms killed earlier."""
    rng = np.random.default_rng({"alpha": 11, "beta": 12, "both": 13}[zero])
    gs = []
    for k in range(3):
        g = synth.random_graph(rng, 24, 16 + k, 12, 2, 2, 16)
        if zero in ("alpha", "both"):
            g.ph_alpha[:] = g.ph_alpha & 4          # class 0, sign bit kept
        if zero in ("beta", "both"):
            g.ph_beta[:] = g.ph_beta & 4
        gs.append(g)
    he = HostEmu(hostemu, gs, 16)
    po = oracle_port.PortOracle(gs, 16)
    for gi, g in enumerate(gs):
        pv = rng.integers(0, 2, size=(48, g.np_params.shape[2])).astype(np.uint8)
        want = po.eval_terms(gi, pv)
        assert np.array_equal(he.eval_terms(gi, pv), want), gi
        assert np.array_equal(he.eval_terms(gi, pv, pairs=True), want), gi
