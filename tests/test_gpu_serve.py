"""Served form: continuous batching through the device-resident request loop.

Each request's bits must be identical to the oracle's and to the plain
one-program call with the same (program, f, seed, rng_mode), whatever else is
in flight: requests are submitted together so their tiles interleave on the
device.  Also: admission by arena footprint (a request larger than the arena
is refused, one that does not fit yet waits and can be cancelled), the loop's
idle exit and relaunch, the side path for wide parameter vectors, and the
device program cache.
"""
from __future__ import annotations

import time

import numpy as np
import pytest

from ksim_b200 import synth

pytestmark = pytest.mark.gpu


def _pool(seed=60):
    rng = np.random.default_rng(seed)
    progs, nfs = [], []
    specs = [(5, 0, 4), (12, 30, 6), (40, 64, 12), (8, 130, 5), (16, 56, 10), (20, 300, 4)]
    for n_out, F, t in specs:                                  # W = 1, 1, 2, 3, 2, 5 (side)
        comp = synth.random_component(rng, n_out=n_out, F=F, t=t, f_prob=0.05)
        progs.append(synth.single_component_program(comp))
        nfs.append(F)
    prog, nf = synth.multi_component_program(rng, [(3, 5, 3), (6, 12, 6), (2, 0, 2)])
    progs.append(prog)
    nfs.append(nf)
    return rng, progs, nfs


@pytest.fixture(scope="module")
def pool():
    return _pool()


def test_served_equals_alone_and_oracle(cuda_device, oracle_port, pool):
    from ksim_b200.sampler import B200ProgramSampler
    from ksim_b200.serve import Server
    rng, progs, nfs = pool
    reqs = []
    for i in range(48):
        pi = int(rng.integers(len(progs)))
        B = int(rng.choice([1, 7, 255, 256, 257, 1000, 3000, 6000]))
        f = synth.sample_f(rng, B, nfs[pi], 0.05)
        reqs.append((pi, f, int(rng.integers(0, 2**63)), int(rng.integers(0, 2))))
    with Server(device=0, idle_us=2000) as srv:
        handles = [srv.submit(progs[pi], f, seed, mode) for pi, f, seed, mode in reqs]
        served = [h.result(timeout=120) for h in handles]
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["side_launches"] > 0 and st["loop_launches"] >= 1
    samplers = [B200ProgramSampler(p, device=0) for p in progs]
    for (pi, f, seed, mode), got in zip(reqs, served):
        alone = samplers[pi].sample(f, seed, rng_mode=mode)
        assert np.array_equal(got, alone)
    for (pi, f, seed, mode), got in list(zip(reqs, served))[::6]:
        assert np.array_equal(got, oracle_port.program_sample(progs[pi], f, seed, rng_mode=mode))


def test_strided_inputs_and_reuse_of_buffers(cuda_device, pool):
    """f given as a row-strided view; the arena is reused across many requests
    (small arena), so stale device data must never leak into a later request."""
    from ksim_b200.sampler import B200ProgramSampler
    from ksim_b200.serve import Server
    rng, progs, nfs = pool
    prog, F = progs[2], nfs[2]
    wide = synth.sample_f(rng, 4000, 128, 0.05)
    alone = B200ProgramSampler(prog, device=0)
    with Server(device=0, arena_bytes=2 << 20, idle_us=500) as srv:
        for rnd in range(3):
            hs = []
            for k in range(12):
                B = int(rng.integers(1, 4000))
                r0 = int(rng.integers(0, 4000 - B + 1))
                f = wide[r0:r0 + B, :F]
                hs.append((f, 100 * rnd + k, srv.submit(prog, f, 100 * rnd + k)))
            for f, seed, h in hs:
                assert np.array_equal(h.result(timeout=120), alone.sample(f, seed))
            time.sleep(0.01)  # let the loop go idle and exit between rounds
        st = srv.stats()
    assert st["loop_launches"] >= 2 and st["completed"] == 36


def test_admission_refusal_wait_and_cancel(cuda_device, pool):
    from ksim_b200._abi import KSIM_ERR_CANCELLED, KsimError
    from ksim_b200.sampler import B200ProgramSampler
    from ksim_b200.serve import Server
    rng, progs, nfs = pool
    prog, F = progs[2], nfs[2]            # 40 outputs, F = 64: 104 bytes per shot
    B = 200_000
    f = synth.sample_f(rng, B, F, 0.05)
    with Server(device=0, arena_bytes=24 << 20) as srv:   # one request fits at a time
        with pytest.raises(MemoryError):
            srv.submit(prog, synth.sample_f(rng, 300_000, F, 0.05), 1)
        first = srv.submit(prog, f, 11)
        second = srv.submit(prog, f, 12)   # waits for the arena
        third = srv.submit(prog, f[:1000], 13)
        second.cancel()
        with pytest.raises(KsimError) as e:
            second.result()
        assert e.value.status == KSIM_ERR_CANCELLED
        got1, got3 = first.result(timeout=120), third.result(timeout=120)
        st = srv.stats()
    s = B200ProgramSampler(prog, device=0)
    assert np.array_equal(got1, s.sample(f, 11))
    assert np.array_equal(got3, s.sample(f[:1000], 13))
    assert st["cancelled"] == 1 and st["completed"] == 2


def test_empty_requests_and_errors(cuda_device, pool):
    from ksim_b200.serve import Server
    rng, progs, nfs = pool
    with Server(device=0) as srv:
        out = srv.submit(progs[1], np.zeros((0, nfs[1]), np.uint8), 3).result()
        assert out.shape == (0, progs[1].num_outputs)
        with pytest.raises(ValueError):
            srv.submit(progs[1], np.zeros((10, nfs[1] - 1), np.uint8), 3)  # too few f columns
        with pytest.raises(TypeError):
            srv.submit(progs[1], np.zeros((10, nfs[1]), np.uint8), -1)


def test_program_cache_lru(cuda_device, pool):
    from ksim_b200.serve import ProgramCache
    _, progs, _ = pool
    cache = ProgramCache(device=0, cache_bytes=1)      # everything unpinned is evicted
    d0, s0 = cache.acquire(progs[0])
    d1, _ = cache.acquire(progs[1])
    assert progs[0] in cache and progs[1] in cache    # both pinned
    cache.release(d1)
    assert progs[1] not in cache and cache.evictions == 1
    d0b, s0b = cache.acquire(progs[0])
    assert d0b == d0 and s0b is s0 and cache.hits == 1
    cache.release(d0)
    cache.release(d0)
    assert len(cache) == 0
