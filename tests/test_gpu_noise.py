"""Device noise draw and device-resident noisy sampling, through the C ABI.

The device draw must equal the oracle's restatement bit for bit (same
counter-based stream), for any shot range; sample_noisy (f drawn and
consumed on the device, chunked) must equal sampling from the oracle-drawn f.
"""
from __future__ import annotations

import numpy as np
import pytest

from ksim_b200 import synth

pytestmark = pytest.mark.gpu


def _model(seed, num_f=40, n_ch=60):
    rng = np.random.default_rng(seed)
    probs = []
    for i in range(n_ch):
        k = int(rng.integers(1, 5))
        p = rng.dirichlet(np.ones(1 << k)) * rng.uniform(1e-3, 0.2)
        p[0] = 1.0 - p[1:].sum()
        probs.append(p)
    n_e = sum(int(np.log2(len(p))) for p in probs)
    T = (rng.random((num_f, n_e)) < 0.1).astype(np.uint8)
    return probs, T


@pytest.mark.parametrize("num_f", [0, 7, 64, 65, 96, 130, 144])
def test_device_draw_equals_oracle(cuda_device, oracle_port, num_f):
    from ksim_b200.noise import DeviceChannelSampler
    probs, T = _model(num_f, num_f=num_f)
    ns = DeviceChannelSampler(probs, T, seed=2**63 + 17)
    for B, off in ((1, 0), (5000, 0), (777, 123456789)):
        got = ns.sample_at(B, off)
        assert np.array_equal(got, oracle_port.noise_sample(probs, T, B, off, 2**63 + 17)), (B, off)
    a, b = ns.sample(300), ns.sample(200)
    assert np.array_equal(np.vstack([a, b]), ns.sample_at(500, 0))


def test_sample_noisy_equals_sampling_the_drawn_f(cuda_device, oracle_port):
    from ksim_b200.noise import DeviceChannelSampler
    from ksim_b200.sampler import B200ProgramSampler
    rng = np.random.default_rng(5)
    prog, n_f = synth.multi_component_program(rng, [(4, 20, 4), (6, 30, 5)])
    probs, T = _model(11, num_f=n_f + 2, n_ch=80)
    ns = DeviceChannelSampler(probs, T, seed=4242)
    s = B200ProgramSampler(prog, device=0)
    for B in (10, 300_001):
        f = ns.sample_at(B, 0)
        assert np.array_equal(f[:2000], oracle_port.noise_sample(probs, T, min(B, 2000), 0, 4242))
        for mode in (0, 1):
            assert np.array_equal(s.sample_noisy(ns, B, 77, rng_mode=mode), s.sample(f, 77, rng_mode=mode))
    with pytest.raises(ValueError):
        s.sample_noisy(DeviceChannelSampler(probs, T[:3], seed=1), 10, 1)


def test_noise_edge_cases(cuda_device, oracle_port):
    """No channels, channels that never fire, no f parameters, and a program
    without f parameters sampled through an empty model."""
    from ksim_b200.noise import DeviceChannelSampler
    from ksim_b200.sampler import B200ProgramSampler
    empty = DeviceChannelSampler([], np.zeros((5, 0), np.uint8), seed=3)
    assert empty.num_channels == 0 and not empty.sample(100).any()
    never = DeviceChannelSampler([np.array([1.0, 0.0]), np.array([1.0, 0, 0, 0])],
                                 np.ones((4, 3), np.uint8), seed=3)
    assert never.num_channels == 0 and not never.sample(100).any()
    nof = DeviceChannelSampler([np.array([0.5, 0.5])], np.zeros((0, 1), np.uint8), seed=3)
    assert nof.sample(10).shape == (10, 0)
    rng = np.random.default_rng(8)
    comp = synth.random_component(rng, n_out=4, F=0, t=4)
    prog = synth.single_component_program(comp)
    s = B200ProgramSampler(prog, device=0)
    assert np.array_equal(s.sample_noisy(nof, 777, 5), s.sample(np.zeros((777, 0), np.uint8), 5))
    assert s.sample_noisy(nof, 0, 5).shape == (0, prog.num_outputs)


def test_device_draw_long_runs_and_merges(cuda_device, oracle_port):
    """A gate-level Pauli model of cfg2's size (8,000 locations, one long run
    of equal firing probability), duplicated signatures that merge, channels
    that always fire and a tiny-probability run: device rows equal the
    oracle's, and the merged model has fewer channels."""
    from ksim_b200.noise import DeviceChannelSampler
    rng = np.random.default_rng(8000)
    probs, T = synth.noise_model(rng, 64, 8000)
    probs = list(probs) + [np.array([1 - 3e-3, 1e-3, 1e-3, 1e-3])] * 50 + [np.array([0.0, 1.0])] * 3 \
        + [np.array([1 - 1e-9, 1e-9])] * 5
    extra = [T[:, :2]] * 50 + [T[:, 2:3]] * 3 + [T[:, 3:4]] * 5
    T = np.hstack([T] + extra)
    ns = DeviceChannelSampler(probs, T, seed=99)
    assert ns.num_channels < len(probs)
    for B, off in ((3000, 0), (1000, 10**9)):
        assert np.array_equal(ns.sample_at(B, off), oracle_port.noise_sample(probs, T, B, off, 99)), (B, off)
