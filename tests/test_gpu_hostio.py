"""Host-buffer sampling: chunked, copy-overlapped calls and bit-packed I/O.

ksim_program_sample splits large calls into chunks of shots (small first and
last chunks, larger ones between) whose copies overlap other chunks'
sampling; each chunk samples with its first
row as shot offset, so the bits must equal one device launch over all shots
(and the oracle).  ksim_program_sample_packed takes and returns rows packed
8 columns per byte; its bits must equal the byte-per-bit call's.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from ksim_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_prog():
    rng = np.random.default_rng(90)
    prog, n_f = synth.multi_component_program(rng, [(3, 9, 3), (5, 14, 4), (2, 0, 2)])
    return rng, prog, n_f


def _device_once(sampler, f, seed, mode):
    import torch
    from ksim_b200 import _abi
    B = f.shape[0]
    d_f = torch.from_numpy(np.ascontiguousarray(f)).cuda()
    d_out = torch.zeros((B, sampler.num_outputs), dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    _abi.check(_abi.lib().ksim_program_sample_device(
        sampler.handle, ctypes.c_void_p(d_f.data_ptr()), B, f.shape[1], 0, seed, mode,
        ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(st)))
    torch.cuda.synchronize()
    return d_out.cpu().numpy()


def _chunk_bounds(B, row_bytes):
    """The host call's chunk schedule (api.cu host_chunk_bounds): u, 2u,
    chunks of about 4u, 2u, u with u ~ B / 32 (>= 16 Ki shots and 256 KiB of
    copies, a multiple of 4 Ki), or chunks of u when B <= 6u."""
    u = (max(1 << 14, B // 32, (1 << 18) // max(row_bytes, 1)) + 4095) // 4096 * 4096
    if B <= 6 * u:
        return list(range(0, B, u)) + [B]
    body = B - 6 * u
    n_body = -(-body // (4 * u))
    step = (body // n_body + 4095) // 4096 * 4096
    return [0, u] + [3 * u + k * step for k in range(n_body)] + [B - 3 * u, B - u, B]


@pytest.mark.parametrize("B", [1, 1000, 65536, 65537, 98305, 131073, 700_001])
def test_chunked_host_call_equals_one_launch(cuda_device, oracle_port, small_prog, B):
    from ksim_b200.sampler import B200ProgramSampler
    rng, prog, n_f = small_prog
    f = synth.sample_f(rng, B, n_f + 3, 0.05)          # extra unused columns
    s = B200ProgramSampler(prog, device=0)
    for mode in (0, 1):
        got = s.sample(f, 31 + B, rng_mode=mode)
        assert np.array_equal(got, _device_once(s, f, 31 + B, mode)), mode
    # spot-check against the oracle across the chunk seams
    bounds = _chunk_bounds(B, f.shape[1] + s.num_outputs)
    assert all(x < y for x, y in zip(bounds, bounds[1:])) and bounds[-1] == B
    got = s.sample(f, 31 + B, rng_mode=1)
    for lo in sorted({max(0, x - 150) for x in bounds}):
        hi = min(B, lo + 300)
        want = oracle_port.program_sample(prog, f[lo:hi], 31 + B, rng_mode=1, shot_offset=lo)
        assert np.array_equal(got[lo:hi], want), lo


@pytest.mark.parametrize("B", [5, 4096, 300_000])
def test_packed_io_equals_byte_io(cuda_device, small_prog, B):
    from ksim_b200.sampler import B200ProgramSampler
    rng, prog, n_f = small_prog
    for extra in (0, 5):
        F = n_f + extra
        f = synth.sample_f(rng, B, F, 0.05)
        s = B200ProgramSampler(prog, device=0)
        want = s.sample(f, 77, rng_mode=0)
        got = s.sample_packed(np.packbits(f, axis=1, bitorder="little"), F, 77, rng_mode=0)
        assert got.shape == (B, (prog.num_outputs + 7) // 8)
        assert np.array_equal(got, np.packbits(want, axis=1, bitorder="little"))
        unpacked = np.unpackbits(got, axis=1, count=prog.num_outputs, bitorder="little")
        assert np.array_equal(unpacked, want)
        into = np.full(got.shape, 0xAB, np.uint8)  # a caller's buffer, filled in place
        assert s.sample_packed(np.packbits(f, axis=1, bitorder="little"), F, 77, rng_mode=0, out=into) is into
        assert np.array_equal(into, got)
    with pytest.raises(ValueError):
        s.sample_packed(np.zeros((3, 1), np.uint8), n_f + 9, 1)
    with pytest.raises(ValueError):
        s.sample_packed(np.zeros((3, (n_f + 7) // 8), np.uint8), n_f, 1, out=np.zeros((2, 1), np.uint8))


def test_packed_io_without_f_columns(cuda_device):
    from ksim_b200.sampler import B200ProgramSampler
    rng = np.random.default_rng(12)
    prog = synth.single_component_program(synth.random_component(rng, n_out=11, F=0, t=3))
    s = B200ProgramSampler(prog, device=0)
    want = s.sample(np.zeros((3001, 0), np.uint8), 9)
    got = s.sample_packed(np.zeros((3001, 0), np.uint8), 0, 9)
    assert np.array_equal(got, np.packbits(want, axis=1, bitorder="little"))
