"""The oracle is pinned before it is trusted.

* the C restatement (oracle/ksim_oracle.c) reproduces, bit for bit, what the
  reference's own zx_eval.hpp produced for the committed fixtures (amplitudes,
  sampled bits and |A_k| for both uniform streams);
* it agrees with the reference's numpy evaluate_flat within 1e-12 relative
  (the reference's own precision gate is 1e-9, tests/test_nonclifford.py:160);
* Philox4x32-10 reproduces the published Random123 known-answer vectors;
* known-answer programs give their closed-form probabilities
  (H T^k H -> sin^2(k pi/8), tests/test_ksim_compile.py:39-49 and
  tests/test_nonclifford.py:105-121; H T H T H -> 1/4, :184-194).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from helpers import golden_names, load_golden, same_bits
from ksim_b200 import synth


@pytest.mark.parametrize("name", golden_names())
def test_port_matches_reference_build_fixtures(oracle_port, name):
    prog, d = load_golden(name)
    for ci, comp in enumerate(prog.components):
        F = int(np.asarray(comp.f_selection).shape[0])
        po = oracle_port.PortOracle(comp.graphs, F)
        for gi in range(len(comp.graphs)):
            pv = d[f"c{ci}_g{gi}_params"]
            assert same_bits(po.eval(gi, pv), d[f"c{ci}_g{gi}_ref_amp"]), (name, gi)
        f = d[f"c{ci}_f"]
        for seed in (11, 2**63 + 12345):
            for mode in (0, 1):
                bits, amp = po.sample(f, seed, mode, return_amp=True)
                assert np.array_equal(bits, d[f"c{ci}_bits_s{seed % 1000}_m{mode}"]), (name, seed, mode)
                assert same_bits(amp, d[f"c{ci}_amp_s{seed % 1000}_m{mode}"]), (name, seed, mode)


@pytest.mark.parametrize("name", [n for n in golden_names() if n != "long"])
def test_port_matches_numpy_evaluate_flat(oracle_port, name):
    prog, d = load_golden(name)
    for ci, comp in enumerate(prog.components):
        F = int(np.asarray(comp.f_selection).shape[0])
        po = oracle_port.PortOracle(comp.graphs, F)
        for gi in range(len(comp.graphs)):
            ours = po.eval(gi, d[f"c{ci}_g{gi}_params"])
            ref = d[f"c{ci}_g{gi}_numpy_amp"]
            scale = max(1e-300, float(np.max(np.abs(ref)))) if ref.size else 1.0
            assert np.max(np.abs(ours - ref), initial=0.0) <= 1e-12 * scale, (name, gi)


@pytest.mark.parametrize("name", [n for n in golden_names() if n != "long"])
def test_port_term_numerators_match_numpy_canonical(oracle_port, name):
    """Same exact Z[w] element per term as numpy's schedule, after both are
    canonicalised (the two evaluators renormalise at different points)."""
    from helpers import canonical_terms
    prog, d = load_golden(name)
    for ci, comp in enumerate(prog.components):
        F = int(np.asarray(comp.f_selection).shape[0])
        po = oracle_port.PortOracle(comp.graphs, F)
        for gi in range(len(comp.graphs)):
            ours = canonical_terms(po.eval_terms(gi, d[f"c{ci}_g{gi}_params"]))
            ref = canonical_terms(d[f"c{ci}_g{gi}_numpy_terms"])
            assert np.array_equal(ours, ref), (name, gi)


def test_port_matches_reference_build_live(oracle_port):
    if not oracle_port.RefOracle.available():
        pytest.skip("oracle/_ref not built on this machine")
    rng = np.random.default_rng(5)
    for trial in range(4):
        n_out, F, t = int(rng.integers(1, 9)), int(rng.integers(0, 70)), int(rng.integers(1, 14))
        comp = synth.random_component(rng, n_out=n_out, F=F, t=t, f_prob=0.05)
        po = oracle_port.PortOracle(comp.graphs, F)
        ro = oracle_port.RefOracle(comp.graphs, F)
        f = synth.sample_f(rng, 300, F, 0.05)
        for mode in (0, 1):
            a, aa = po.sample(f, 99 + trial, mode, return_amp=True)
            b, bb = ro.sample(f, 99 + trial, mode, return_amp=True)
            assert np.array_equal(a, b) and same_bits(aa, bb)


def test_philox_known_answers(oracle_port):
    # Random123 kat_vectors, philox4x32 with 10 rounds
    cases = [
        ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]
    for ctr, key, want in cases:
        assert oracle_port.philox4x32_10(ctr, key) == want


def test_exp2_of_integers_is_exact(oracle_port):
    """The complex cast scales by exp2(integer); the kernels build 2^n
    directly, which equals libm's exp2 on every representable exponent."""
    for n in range(-1074, 1024):
        assert oracle_port.exp2_int(n) == math.ldexp(1.0, n)
    assert oracle_port.exp2_int(-1075) == 0.0
    assert math.isinf(oracle_port.exp2_int(1024))


@pytest.mark.parametrize("k", [1, 2, 3, 5, 7])
def test_htkh_exact_probability(oracle_port, k):
    prog, exact = synth.htkh(k)
    comp = prog.components[0]
    po = oracle_port.PortOracle(comp.graphs, 0)
    p1 = po.eval_abs(1, np.ones((1, 1), np.uint8))[0]
    p0 = po.eval_abs(0, np.zeros((1, 0), np.uint8))[0]
    assert abs(p1 / p0 - exact) < 1e-15


def test_htkh_sampled_frequency(oracle_port):
    for k in (1, 2, 3):
        prog, exact = synth.htkh(k)
        n = 20_000
        bits = oracle_port.program_sample(prog, np.zeros((n, 0), np.uint8), seed=11)
        sigma = math.sqrt(exact * (1 - exact) / n)
        assert abs(bits[:, 0].mean() - exact) < 5 * sigma


def test_t_depth_two(oracle_port):
    prog, exact = synth.t_depth_two()
    comp = prog.components[0]
    po = oracle_port.PortOracle(comp.graphs, 0)
    assert abs(po.eval_abs(1, np.ones((1, 1), np.uint8))[0] - exact) < 1e-15
    n = 20_000
    bits = oracle_port.program_sample(prog, np.zeros((n, 0), np.uint8), seed=11)
    assert abs(bits[:, 0].mean() - exact) < 5 * math.sqrt(exact * (1 - exact) / n)


def test_mixture_marginals_exact(oracle_port):
    rng = np.random.default_rng(21)
    prog, F, prob = synth.mixture(rng, n_out=4, r=2, F=2)
    comp = prog.components[0]
    po = oracle_port.PortOracle(comp.graphs, F)
    for f in ([0, 0], [1, 0], [0, 1], [1, 1]):
        for m in range(16):
            bits = [(m >> j) & 1 for j in range(4)]
            # graph 4 holds P(m0..m2, m3 = 1); by symmetry use the full outcome with m3 = 1
            if bits[3] != 1:
                continue
            params = np.array([f + bits[:3] + [1]], np.uint8)
            got = po.eval_abs(4, params)[0]
            assert abs(got - prob(f, bits)) < 1e-14


def test_mixture_sampled_distribution(oracle_port):
    rng = np.random.default_rng(22)
    prog, F, prob = synth.mixture(rng, n_out=3, r=2, F=1)
    n = 40_000
    f = np.zeros((n, 1), np.uint8)
    bits = oracle_port.program_sample(prog, f, seed=5, rng_mode=1)
    codes = bits[:, 0] + 2 * bits[:, 1] + 4 * bits[:, 2]
    counts = np.bincount(codes, minlength=8)
    for m in range(8):
        p = prob([0], [(m >> j) & 1 for j in range(3)])
        sigma = math.sqrt(max(p * (1 - p), 1e-12) / n)
        assert abs(counts[m] / n - p) < 5 * sigma + 1e-12
