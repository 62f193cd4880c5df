"""``sample_compiled`` / ``sample_circuit``: the post-compile part of ksim.sample_circuit.

Reference: src/python/ksim/run.py:45-91.  With a noiseless model f is all
zero (run.py:70-72), so (det, obs) must be the reference kernel's bits
(``oracle/_ref``) split at num_detectors.  With a noise model the f rows are
drawn on the device; the result must equal sampling the oracle's
restatement of that draw (``oracle.noise_sample``, same counter-based stream)
with the reference kernel.  The distribution of the draw itself is pinned to
the reference's ChannelSampler in tests/test_noise.py.
"""
from __future__ import annotations

import numpy as np
import pytest

from ksim_b200 import synth

pytestmark = pytest.mark.gpu


def _program(num_detectors=7):
    rng = np.random.default_rng(6060)
    prog, n_f = synth.multi_component_program(rng, [(5, 12, 5), (6, 20, 6)])
    prog.num_detectors = num_detectors
    return prog, n_f, rng


def test_noiseless_split_at_num_detectors(cuda_device, oracle_module, ref_oracle):
    from ksim_b200.run import sample_compiled
    rng = np.random.default_rng(6161)
    prog, _ = synth.multi_component_program(rng, [(5, 0, 5), (6, 0, 6)])  # no f parameters
    prog.num_detectors = 7
    det, obs = sample_compiled(prog, [], np.zeros((0, 0), np.uint8), 3000, seed=99)
    want = oracle_module.program_sample(prog, np.zeros((3000, 0), np.uint8), 99, 0, oracle_cls=ref_oracle)
    assert det.dtype == np.uint8 and obs.dtype == np.uint8
    assert det.shape == (3000, 7) and obs.shape == (3000, prog.num_outputs - 7)
    assert np.array_equal(np.hstack([det, obs]), want)
    # an empty model for a program that reads f columns: f has no columns
    # (run.py:70-72) and the f_selection gather fails, as in the reference
    noisy_prog, n_f, _ = _program()
    with pytest.raises(IndexError):
        sample_compiled(noisy_prog, [], np.zeros((n_f, 0), np.uint8), 10, seed=1)


@pytest.mark.parametrize("mode", [0, 1])
def test_noisy_equals_sampling_the_drawn_f(cuda_device, oracle_module, ref_oracle, mode):
    from ksim_b200.run import sample_compiled
    prog, n_f, rng = _program()
    probs, T = synth.noise_model(rng, n_f, 300, p=5e-3)
    det, obs = sample_compiled(prog, probs, T, 4000, seed=123, rng_mode=mode)
    f = oracle_module.noise_sample(probs, T, 4000, 0, 123)
    want = oracle_module.program_sample(prog, f, 123, mode, oracle_cls=ref_oracle)
    assert np.array_equal(np.hstack([det, obs]), want)


def test_sample_circuit_with_a_compile_step_and_reused_sampler(cuda_device):
    from ksim_b200.run import sample_circuit, sample_compiled
    from ksim_b200.sampler import B200ProgramSampler
    prog, n_f, rng = _program(num_detectors=0)
    probs, T = synth.noise_model(rng, n_f, 50)
    seen = []

    def compile_fn(circuit):
        seen.append(circuit)
        return prog, probs, T

    det, obs = sample_circuit("H 0\nT 0\nH 0\nM 0", 500, compile_fn=compile_fn, seed=5, backend="gpu")
    assert seen == ["H 0\nT 0\nH 0\nM 0"] and det.shape == (500, 0) and obs.shape == (500, prog.num_outputs)
    s = B200ProgramSampler(prog, device=0)
    d2, o2 = sample_compiled(prog, probs, T, 500, seed=5, sampler=s, backend="auto")
    assert np.array_equal(o2, obs) and d2.shape == (500, 0)
