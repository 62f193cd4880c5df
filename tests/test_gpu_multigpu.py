"""The shot-split multi-GPU sampler on one GPU, through its device sampler.

``ShardedSampler`` without a process group is world size 1: its
``_device_sampler`` (``ksim_program_sample_device`` with ``shot_offset``)
must return the oracle's bits.  The rank arithmetic of larger worlds is then
replayed on the same GPU one rank after another (``sample_local`` only, no
collective and no rank waiting on another): the concatenated slices must be
the one-call result, because every uniform is keyed by the absolute shot
index.  The gather over a real process group is covered by the gloo tests
(``tests/test_multirank.py``).
"""
from __future__ import annotations

import numpy as np
import pytest

from ksim_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [0, 1])
def test_sharded_sampler_world1_and_replayed_ranks(cuda_device, oracle_module, ref_oracle, mode):
    from ksim_b200.multigpu import ShardedSampler
    rng = np.random.default_rng(8080 + mode)
    prog, n_f = synth.multi_component_program(rng, [(6, 20, 6), (9, 30, 8)])
    f = synth.sample_f(rng, 5001, n_f, 0.04)
    want = oracle_module.program_sample(prog, f, 4321, mode, oracle_cls=ref_oracle)
    ss = ShardedSampler(prog, device=0)
    assert ss.world == 1 and ss.rank == 0
    assert np.array_equal(ss.sample(f, 4321, rng_mode=mode), want)
    for world in (2, 3, 8):
        parts = []
        for rank in range(world):
            ss.world, ss.rank = world, rank
            lo, hi, bits = ss.sample_local(f, 4321, rng_mode=mode)
            parts.append((lo, hi, bits))
        assert [p[0] for p in parts] == sorted(p[0] for p in parts)
        got = np.concatenate([b for _, _, b in parts], axis=0)
        assert got.shape == want.shape and np.array_equal(got, want), world
