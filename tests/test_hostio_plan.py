"""The chunk plan of host-buffer sampling calls (ksim_b200/csrc/hostio.h), on the CPU.

ksim_program_sample (and its packed and noisy forms, and Component.sample)
samples B shots in chunks so that copies overlap sampling; each chunk samples
with shot_offset = its first row, so any plan gives the bits of one launch
(the GPU tests check the seams against the oracle).  Here the plan itself:
it covers [0, B) with increasing boundaries, ramps up and down, keeps chunks
large enough to repay their launches, and the output-copy lag stays within
the compute streams.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest


@pytest.fixture(scope="module")
def plan(hostemu):
    L = hostemu
    L.hostemu_chunk_bounds.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64),
                                       ctypes.c_int]
    L.hostemu_chunk_bounds.restype = ctypes.c_int
    L.hostemu_copy_lag.argtypes = [ctypes.POINTER(ctypes.c_int64), ctypes.c_int, ctypes.c_int64, ctypes.c_int]
    L.hostemu_copy_lag.restype = ctypes.c_int

    def bounds(B, row_bytes):
        out = (ctypes.c_int64 * 256)()
        n = L.hostemu_chunk_bounds(B, row_bytes, out, 256)
        assert 0 < n <= 256
        return list(out[:n])

    def lag(b, wave, max_lag=4):
        arr = (ctypes.c_int64 * len(b))(*b)
        return L.hostemu_copy_lag(arr, len(b), wave, max_lag)

    return bounds, lag


SIZES = [1, 7, 4096, 16383, 16384, 16385, 65536, 98304, 98305, 131073, 300_001, 700_001, 1_000_000,
         4_000_000, 10_000_001, 123_456_789]


@pytest.mark.parametrize("row_bytes", [0, 1, 5, 13, 104, 168, 4096])
def test_plan_covers_the_shots_in_order(plan, row_bytes):
    bounds, _ = plan
    for B in SIZES:
        b = bounds(B, row_bytes)
        assert b[0] == 0 and b[-1] == B, (B, row_bytes)
        assert all(x < y for x, y in zip(b, b[1:])), (B, row_bytes, b)
        # inner boundaries on 4 Ki shots (the last one before B may not be)
        u = max(1 << 14, B // 32, (1 << 18) // max(row_bytes, 1))
        u = (u + 4095) // 4096 * 4096
        sizes = np.diff(b)
        if B <= 6 * u:
            assert all(s == u for s in sizes[:-1]) and sizes[-1] <= u, (B, row_bytes)
        else:
            # the ramp: u, 2u up front, 2u, u at the end, about 4u between
            assert list(sizes[:2]) == [u, 2 * u] and list(sizes[-2:]) == [2 * u, u], (B, row_bytes)
            body = sizes[2:-2]
            assert len(body) >= 1 and all(0 < s <= 4 * u + 4096 for s in body), (B, row_bytes, body)


def test_small_copies_get_few_chunks(plan):
    """A chunk moves at least 256 KiB across PCIe when the call has that much."""
    bounds, _ = plan
    b = bounds(100_000, 5)               # cfg1: 5 output bytes a shot, no f
    assert len(b) - 1 == 2
    for B, rb in ((1_000_000, 104), (1_000_000, 13), (300_001, 168)):
        sizes = np.diff(bounds(B, rb))
        assert all(s * rb >= (1 << 18) for s in sizes[:-1]), (B, rb)


def test_copy_lag_fills_a_wave_within_the_streams(plan):
    bounds, lag = plan
    wave = 148 * 5 * 256
    assert lag(bounds(1_000_000, 104), wave) == 2      # chunks of ~118 Ki shots
    assert lag(bounds(50_000, 168), wave) == 4         # 16 Ki-shot chunks: capped at the streams
    assert lag([0, 10**8], wave) == 1                  # one chunk larger than a wave
    for B in SIZES:
        assert 1 <= lag(bounds(B, 104), wave) <= 4
