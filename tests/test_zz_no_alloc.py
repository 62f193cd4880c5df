"""The allocation-free sampling entry point against the regular one.

``ksim_component_sample_device_noalloc`` is for callers that cannot allocate
device memory: their HBM belongs to another allocator or is reserved up front,
or a cudaMalloc / cudaFree (which may synchronise the whole device) is not
allowed inside their sampling loop.  It keeps its scratch in a fixed device
array inside the library.  Here it must return exactly the bits and |A_k| of
``ksim_component_sample_device`` (bit-exact, the tolerance of every parity
test in this suite) on two calls in a row, so the scratch one call leaves
behind does not leak into the next, and the second call must take no device
memory.  The file sorts last so that a run stopping at the first failure has
run every other test before it.
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
