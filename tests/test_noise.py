"""The noise draw (f parameters) against the reference's ChannelSampler, on the CPU.

Fixtures (tests/golden/noise_*.npz, made by make_noise_golden.py from the
reference's compile/channels.py) hold, for three noise models built with the
reference's own channel constructors, the exact probability of seeded parity
sets of f computed from the reference's precomputed (simplified) channels and
the parity frequencies of 200,000 reference draws.

* the model here (unsimplified channels, exact parity formula) gives the
  reference's exact parity probabilities to 1e-12 — the distribution of f is
  pinned to the reference's;
* the oracle's restatement of the device draw hits every exact probability
  within 5 sigma on 200,000 shots, as do the reference's own draws.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from ksim_b200.noise import parity_probability

GOLDEN = ["flips", "pauli1", "pauli2_heralded"]


def load(name):
    from pathlib import Path
    d = np.load(Path(__file__).parent / "golden" / f"noise_{name}.npz")
    n_bits = d["n_bits"]
    probs, off = [], 0
    for k in n_bits:
        probs.append(d["probs"][off:off + (1 << int(k))])
        off += 1 << int(k)
    sets, off = [], 0
    for n in d["set_len"]:
        sets.append(d["set_cols"][off:off + int(n)].tolist())
        off += int(n)
    return probs, d["transform"], sets, d["exact"], d["ref_freq"], int(d["ref_shots"])


def _within(freq, p, n, sig=5.0):
    sd = math.sqrt(max(p * (1 - p), 1e-12) / n)
    return abs(freq - p) <= sig * sd + 1e-9


@pytest.mark.parametrize("name", GOLDEN)
def test_exact_parities_match_reference(name):
    probs, T, sets, exact, _, _ = load(name)
    for s, want in zip(sets, exact):
        assert abs(parity_probability(probs, T, s) - want) <= 1e-12, s


@pytest.mark.parametrize("name", GOLDEN)
def test_reference_draws_hit_exact(name):
    _, _, sets, exact, freq, n = load(name)
    for s, p, fr in zip(sets, exact, freq):
        assert _within(fr, p, n), (s, p, fr)


@pytest.mark.parametrize("name", GOLDEN)
def test_oracle_draw_hits_exact(oracle_port, name):
    probs, T, sets, exact, _, _ = load(name)
    n = 200_000
    f = oracle_port.noise_sample(probs, T, n, 0, 12345)
    assert f.shape == (n, T.shape[0]) and f.max() <= 1
    for s, p in zip(sets, exact):
        assert _within(float((f[:, s].sum(axis=1) % 2).mean()), p, n), (s, p)


def test_oracle_draw_is_counter_based(oracle_port):
    probs, T, _, _, _, _ = load("pauli1")
    full = oracle_port.noise_sample(probs, T, 3000, 0, 99)
    part = oracle_port.noise_sample(probs, T, 1000, 1500, 99)
    assert np.array_equal(full[1500:2500], part)
    assert not np.array_equal(full, oracle_port.noise_sample(probs, T, 3000, 0, 100))


def test_model_validation():
    from ksim_b200.noise import _model_arrays
    with pytest.raises(ValueError):
        _model_arrays([np.array([0.5, 0.3, 0.2])], np.zeros((2, 2), np.uint8))
    with pytest.raises(ValueError):
        _model_arrays([np.array([0.9, 0.1])], np.zeros((2, 3), np.uint8))


def test_merged_channels_and_long_runs_hit_exact(oracle_port):
    """Channels over identical error-bit patterns are merged by XOR
    convolution, and equal firing probabilities share one skip table: the
    draw must still follow the model's exact parity probabilities (computed
    from the unmerged channels)."""
    rng = np.random.default_rng(31)
    num_f = 12
    sigs = [rng.integers(0, 2, size=(num_f, 2)).astype(np.uint8) for _ in range(15)]
    probs, cols = [], []
    for i in range(240):                       # 16 copies of each signature pair
        probs.append(np.array([1 - 3e-2, 1e-2, 1e-2, 1e-2]))
        cols.append(sigs[i % 15])
    for i in range(40):                        # one-bit channels, some never-firing
        probs.append(np.array([1.0, 0.0]) if i % 7 == 0 else np.array([0.98, 0.02]))
        cols.append(rng.integers(0, 2, size=(num_f, 1)).astype(np.uint8))
    T = np.hstack(cols)
    n = 200_000
    f = oracle_port.noise_sample(probs, T, n, 0, 777)
    sets = [[j] for j in range(num_f)] + [[0, 3], [1, 5, 7], [2, 4, 6, 8]]
    for s in sets:
        p = parity_probability(probs, T, s)
        assert _within(float((f[:, s].sum(axis=1) % 2).mean()), p, n), (s, p)
