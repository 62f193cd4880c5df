"""Host-side bookkeeping of the sampling server, on the CPU.

The arena that admits requests by HBM footprint and the admission rule
(``ksim_b200/csrc/serve_sched.h``) run here through the host-compiled test
shim: random alloc / release scripts against a model of the free space, and
the admit / wait / never-fits decisions.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest


@pytest.fixture(scope="module")
def shim(hostemu):
    L = hostemu
    i64p = ctypes.POINTER(ctypes.c_int64)
    L.hostemu_arena_run.argtypes = [ctypes.c_int64, ctypes.c_int64, i64p, ctypes.c_int, i64p, i64p]
    L.hostemu_arena_run.restype = None
    L.hostemu_admissible.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.c_int64, ctypes.c_int64,
                                     ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int64, ctypes.c_int64]
    L.hostemu_admissible.restype = ctypes.c_int
    return L


def _run(L, cap, align, ops):
    ops = np.ascontiguousarray(np.asarray(ops, np.int64).reshape(-1, 2))
    res = np.zeros(len(ops), np.int64)
    state = np.zeros(4, np.int64)
    p = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))  # noqa: E731
    L.hostemu_arena_run(cap, align, p(ops), len(ops), p(res), p(state))
    return res, state


@pytest.mark.parametrize("seed", range(6))
def test_arena_random_scripts(shim, seed):
    rng = np.random.default_rng(seed)
    cap, align = 1 << 20, 256
    ops, live = [], []
    for i in range(400):
        if live and rng.random() < 0.45:
            k = live.pop(int(rng.integers(len(live))))
            ops.append((1, k))
        else:
            ops.append((0, int(rng.integers(1, 60000))))
            live.append(i)
    res, state = _run(shim, cap, align, ops)
    # replay: blocks never overlap, stay aligned and inside the arena
    blocks = {}
    for i, (kind, arg) in enumerate(ops):
        if kind == 0:
            off = int(res[i])
            if off < 0:
                continue
            size = -(-arg // align) * align
            assert off % align == 0 and 0 <= off and off + size <= cap
            for o, sz in blocks.values():
                assert off + size <= o or o + sz <= off, "overlap"
            blocks[i] = (off, size)
        else:
            was_live = arg in blocks
            assert res[i] == (1 if was_live else 0)
            blocks.pop(arg, None)
    assert state[0] == sum(sz for _, sz in blocks.values())
    assert state[3] == len(blocks)
    # releasing everything merges back into one block of the whole arena
    ops2 = list(ops) + [(1, i) for i in blocks]
    _, state2 = _run(shim, cap, align, ops2)
    assert state2.tolist() == [0, cap, 1, 0]


def test_arena_first_fit_and_merge(shim):
    ops = [(0, 100), (0, 300), (0, 256), (1, 1), (0, 200), (0, 600)]
    res, state = _run(shim, 2048, 256, ops)
    assert res[:3].tolist() == [0, 256, 768]
    assert res[3] == 1
    assert res[4] == 256          # first fit reuses the freed 512-byte hole
    assert res[5] == 1024         # 768 bytes do not fit the 256-byte remainder of the hole
    assert res[0] >= 0 and state[3] == 4
    res, _ = _run(shim, 1024, 256, [(0, 2000)])
    assert res[0] == -1


def test_admission_rule(shim):
    A = shim.hostemu_admissible
    MB = 1 << 20
    # fits now
    assert A(MB, 2, 2, 8 * MB, 0, 4, 4, 8, 8, 16, 0) == 1
    # larger than the whole arena / job table / ring: never
    assert A(9 * MB, 1, 1, 8 * MB, 0, 4, 4, 8, 8, 16, 0) == -1
    assert A(MB, 9, 9, 8 * MB, 0, 4, 4, 8, 8, 16, 0) == -1
    assert A(MB, 2, 17, 8 * MB, 0, 4, 4, 8, 8, 16, 0) == -1
    # waits: arena busy, no request slot, too few job slots, ring full
    assert A(4 * MB, 1, 1, 8 * MB, 5 * MB, 4, 4, 8, 8, 16, 0) == 0
    assert A(MB, 1, 1, 8 * MB, 0, 0, 4, 8, 8, 16, 0) == 0
    assert A(MB, 3, 3, 8 * MB, 0, 4, 4, 2, 8, 16, 0) == 0
    assert A(MB, 2, 2, 8 * MB, 0, 4, 4, 8, 8, 16, 15) == 0
    assert A(MB, 2, 2, 8 * MB, 0, 4, 4, 8, 8, 16, 14) == 1
