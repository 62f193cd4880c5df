"""Failure detection on the device: a staging wait that runs out.

Every mbarrier wait of the sampling kernels is bounded.  With the component's
wait bound set to one non-blocking poll, the first wait of a CTA (its first
chunk's copy was issued a moment earlier) gives up while the copy is still in
flight: the CTA raises KSIM_FLAG_WAIT_TIMEOUT, waits with the built-in bound
for the copies it issued (they land), and leaves without writing its shots.
Nothing faults or hangs: the copy completes, the kernel returns, and the same
context then samples correctly.  Reference error path: kokkos_sim.cpp:193-194
(the reference has no bounded waits; its only reported error is the
argument check).
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from ksim_b200 import synth

pytestmark = pytest.mark.gpu


def _component(seed=910):
    from ksim_b200.kokkos_sim import Component
    rng = np.random.default_rng(seed)
    comp = synth.random_component(rng, n_out=20, F=60, t=12, f_prob=0.05)
    kc = Component(comp.graphs, 60)
    f = synth.sample_f(rng, 20000, 60, 0.05)
    return comp, kc, f


def test_plain_wait_timeout_is_reported_and_context_survives(cuda_device, oracle_port):
    from ksim_b200._abi import FLAG_WAIT_TIMEOUT
    comp, kc, f = _component()
    assert kc.get_launch()["staged"] == 1
    want = oracle_port.PortOracle(comp.graphs, 60).sample(f, 5, 0)
    kc.set_wait_limit(1)
    with pytest.raises(TimeoutError, match="staging wait"):
        kc.sample(f, 5)
    # the host call consumed the flag it reported
    assert not kc.status() & FLAG_WAIT_TIMEOUT

    # on device buffers the flag stays in the component's status word
    import torch
    from ksim_b200 import _abi
    d_f = torch.from_numpy(f).cuda()
    d_out = torch.full((f.shape[0], kc.n_out), 9, dtype=torch.uint8, device="cuda")
    _abi.check(_abi.lib().ksim_component_sample_device(
        kc.handle, ctypes.c_void_p(d_f.data_ptr()), f.shape[0], 0, 5, 0,
        ctypes.c_void_p(d_out.data_ptr()), kc.n_out, 0, None,
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    assert kc.status(reset=True) & FLAG_WAIT_TIMEOUT
    assert (d_out.cpu().numpy() == 9).any(), "a CTA that gave up must not write its shots"

    # back to the built-in bound: same context, exact results
    kc.set_wait_limit(0)
    assert np.array_equal(kc.sample(f, 5), want)
    assert kc.status() == 0


def test_program_call_reports_a_wait_timeout(cuda_device, oracle_port):
    """The pipelined host call of a program reads its components' status
    words behind its last output copy: a wait that ran out fails the call
    (and leaves the word clear), and the next call is exact."""
    from ksim_b200._abi import FLAG_WAIT_TIMEOUT
    from ksim_b200.sampler import B200ProgramSampler
    comp, _, f = _component()
    prog = synth.single_component_program(comp)
    s = B200ProgramSampler(prog, device=0)
    kc = s.components[0][1]
    kc.set_wait_limit(1)
    with pytest.raises(TimeoutError, match="staging wait"):
        s.sample(f, 5)
    assert not kc.status() & FLAG_WAIT_TIMEOUT
    kc.set_wait_limit(0)
    assert np.array_equal(s.sample(f, 5), oracle_port.program_sample(prog, f, 5))


def test_served_wait_timeout_fails_the_request_only(cuda_device, oracle_port):
    from ksim_b200.serve import Server
    comp, _, f = _component(911)
    prog = synth.single_component_program(comp)
    want = oracle_port.program_sample(prog, f[:3000], 77, 1)
    with Server(device=0, idle_us=2000) as srv:
        d, sampler = srv.cache.acquire(prog)
        for _, kc in sampler.components:
            kc.set_wait_limit(1)
        bad = srv.submit(prog, f, 76, 1)
        with pytest.raises(TimeoutError, match="wait"):
            bad.result(timeout=120)
        for _, kc in sampler.components:
            kc.set_wait_limit(0)
        srv.cache.release(d)
        good = srv.submit(prog, f[:3000], 77, 1)
        assert np.array_equal(good.result(timeout=120), want)
        st = srv.stats()
    assert st["failed"] == 1 and st["completed"] == 1
