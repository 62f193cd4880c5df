"""The allocation-free sampling entry point against the regular one.

``ksim_component_sample_device_noalloc`` is for callers that cannot allocate
device memory: their HBM belongs to another allocator or is reserved up front,
or a cudaMalloc / cudaFree (which may synchronise the whole device) is not
allowed inside their sampling loop.  It keeps its scratch (the staging chunk
directory) in a fixed device array inside the library.  Here it must return
exactly the bits and |A_k| of ``ksim_component_sample_device`` (bit-exact,
the tolerance of every parity test in this suite) on two calls in a row, so
the scratch one call leaves behind does not leak into the next, for the
staged and the unstaged launch and for a wide (W > 4) parameter vector; the
kernel's status flags must reach ``ksim_component_status``; and the call must
take no device memory.  The file sorts last so that a run stopping at the
first failure has run every other test before it.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from ksim_b200 import synth

pytestmark = pytest.mark.gpu


def _call(fn, kc, d_f, B, offset, seed, mode, d_out, d_amp, stream):
    from ksim_b200 import _abi
    _abi.check(fn(kc.handle, ctypes.c_void_p(d_f.data_ptr()), B, offset, seed, mode,
                  ctypes.c_void_p(d_out.data_ptr()), d_out.shape[1], 0,
                  ctypes.c_void_p(d_amp.data_ptr()), ctypes.c_void_p(stream)))


def _same_as_sample_device(kc, F, rng, B=4000):
    """Two calls in a row of each entry point on the same inputs; bits and
    |A_k| compared bit for bit."""
    import torch
    from ksim_b200 import _abi
    L = _abi.lib()
    d_f = torch.from_numpy(synth.sample_f(rng, B, F, 0.05)).cuda()
    shape_out, shape_amp = (B, kc.n_out), (B, kc.n_out + 1)
    ref_out = torch.zeros(shape_out, dtype=torch.uint8, device="cuda")
    ref_amp = torch.zeros(shape_amp, dtype=torch.float64, device="cuda")
    out = torch.full(shape_out, 7, dtype=torch.uint8, device="cuda")
    amp = torch.full(shape_amp, -1.0, dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    for seed, mode, offset in ((123, 0, 0), (2**63 + 5, 1, 777)):
        _call(L.ksim_component_sample_device, kc, d_f, B, offset, seed, mode, ref_out, ref_amp, st)
        _call(L.ksim_component_sample_device_noalloc, kc, d_f, B, offset, seed, mode, out, amp, st)
        torch.cuda.synchronize()
        assert torch.equal(out, ref_out), (seed, mode)
        assert np.array_equal(amp.cpu().numpy().view(np.uint64),
                              ref_amp.cpu().numpy().view(np.uint64)), (seed, mode)


@pytest.mark.parametrize("staged", [1, 0])
def test_noalloc_unstaged_and_wide_vectors(cuda_device, staged):
    from ksim_b200.kokkos_sim import Component
    rng = np.random.default_rng(4343 + staged)
    comp = synth.random_component(rng, n_out=7, F=300, t=6, f_prob=0.02)  # 308 bits: W = 5
    kc = Component(comp.graphs, 300)
    assert kc.words > 4
    kc.set_launch(staged=staged)
    _same_as_sample_device(kc, 300, rng, B=1500)


def test_noalloc_flags_reach_the_component_status(cuda_device):
    import torch
    from ksim_b200 import _abi
    from ksim_b200._abi import FLAG_INT64_RISK, FLAG_WAIT_TIMEOUT
    from ksim_b200.kokkos_sim import Component
    from ksim_b200.program import FlatComponent
    L = _abi.lib()
    st = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(250)
    # 250 NodePhases factors (1 + w^(1+4 par)): the exact path wraps int64
    gs = [synth.random_graph(rng, 3, 20 + k, 250, 3, 3, 40) for k in range(4)]
    for g in gs:
        g.np_phases[:] = 1
        g.np_params[:] = 0
        g.np_params[:, ::7, 0] = 1
        g.np_counts[:] = 250
    kc = Component(FlatComponent((0, 1, 2), np.arange(20, dtype=np.int32), gs).graphs, 20)
    d_f = torch.from_numpy(synth.sample_f(rng, 256, 20, 0.1)).cuda()
    out = torch.zeros((256, 3), dtype=torch.uint8, device="cuda")
    amp = torch.zeros((256, 4), dtype=torch.float64, device="cuda")
    assert kc.status(reset=True) == 0
    _call(L.ksim_component_sample_device_noalloc, kc, d_f, 256, 0, 3, 0, out, amp, st)
    torch.cuda.synchronize()
    assert kc.status(reset=True) & FLAG_INT64_RISK

    # a staging wait bounded to one poll gives up, and the flag is visible
    comp = synth.random_component(rng, n_out=20, F=60, t=12, f_prob=0.05)
    kc2 = Component(comp.graphs, 60)
    kc2.set_wait_limit(1)
    B = 20000
    d_f = torch.from_numpy(synth.sample_f(rng, B, 60, 0.05)).cuda()
    out = torch.zeros((B, 20), dtype=torch.uint8, device="cuda")
    amp = torch.zeros((B, 21), dtype=torch.float64, device="cuda")
    _call(L.ksim_component_sample_device_noalloc, kc2, d_f, B, 0, 3, 0, out, amp, st)
    torch.cuda.synchronize()
    assert kc2.status(reset=True) & FLAG_WAIT_TIMEOUT
    kc2.set_wait_limit(0)


def test_noalloc_entry_point_matches_sample_device(cuda_device):
    import torch
    from ksim_b200 import _abi
    from ksim_b200.kokkos_sim import Component
    L = _abi.lib()
    rng = np.random.default_rng(4242)
    comp = synth.random_component(rng, n_out=9, F=70, t=10, f_prob=0.05)  # 79 bits: W = 2
    F = int(np.asarray(comp.f_selection).shape[0])
    kc = Component(comp.graphs, F)
    B = 4000
    d_f = torch.from_numpy(synth.sample_f(rng, B, F, 0.05)).cuda()
    shape_out, shape_amp = (B, kc.n_out), (B, kc.n_out + 1)
    ref_out = torch.zeros(shape_out, dtype=torch.uint8, device="cuda")
    ref_amp = torch.zeros(shape_amp, dtype=torch.float64, device="cuda")
    out = torch.full(shape_out, 7, dtype=torch.uint8, device="cuda")
    amp = torch.full(shape_amp, -1.0, dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream

    for seed, mode, offset in ((123, 0, 0), (2**63 + 5, 1, 777)):
        _call(L.ksim_component_sample_device, kc, d_f, B, offset, seed, mode, ref_out, ref_amp, st)
        _call(L.ksim_component_sample_device_noalloc, kc, d_f, B, offset, seed, mode, out, amp, st)
        torch.cuda.synchronize()
        assert torch.equal(out, ref_out), (seed, mode)
        assert np.array_equal(amp.cpu().numpy().view(np.uint64),
                              ref_amp.cpu().numpy().view(np.uint64)), (seed, mode)

    free_before = torch.cuda.mem_get_info()[0]
    _call(L.ksim_component_sample_device_noalloc, kc, d_f, B, 0, 9, 0, out, amp, st)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before


def test_noalloc_rejects_a_component_beyond_the_scratch(cuda_device):
    import torch
    from ksim_b200 import _abi
    from ksim_b200.kokkos_sim import Component
    L = _abi.lib()
    rng = np.random.default_rng(7)
    # 3000 terms, a staging slot of the largest term: at least 1500 chunks, more
    # than the scratch holds (two terms share a chunk at most)
    gs = [synth.random_graph(rng, 3000 if k == 1 else 2, 6 + k, 8, 2, 2, 2) for k in range(3)]
    kc = Component(gs, 6)
    kc.set_launch(slot_bytes=(kc.stats()["max_term_bytes"] + 15) // 16 * 16)
    d_f = torch.zeros((64, 6), dtype=torch.uint8, device="cuda")
    out = torch.zeros((64, 2), dtype=torch.uint8, device="cuda")
    amp = torch.zeros((64, 3), dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    with pytest.raises(_abi.KsimError) as e:
        _call(L.ksim_component_sample_device_noalloc, kc, d_f, 64, 0, 1, 0, out, amp, st)
    assert e.value.status == _abi.KSIM_ERR_UNSUPPORTED and "1024" in str(e.value)
