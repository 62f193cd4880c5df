"""Helpers shared by the tests (fixture loading, host-emulator calls)."""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from ksim_b200._abi import graphs_to_descs
from ksim_b200.program import graph_to_dict, load_program

GOLDEN = Path(__file__).resolve().parent / "golden"


def golden_names() -> list:
    return [n.strip() for n in (GOLDEN / "MANIFEST.txt").read_text().split() if n.strip()]


def load_golden(name: str):
    prog = load_program(GOLDEN / f"prog_{name}.npz")
    data = np.load(GOLDEN / f"golden_{name}.npz")
    return prog, data


def same_bits(a: np.ndarray, b: np.ndarray) -> bool:
    """Bit-identical float arrays (NaNs compared by pattern)."""
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def complex_pairs(z: np.ndarray) -> np.ndarray:
    return np.stack([np.real(z), np.imag(z)], axis=-1).astype(np.float64)


class HostEmu:
    """The device term evaluator compiled for the CPU (tests only)."""

    def __init__(self, L, graphs, F):
        self.L = L
        self.graphs = [g if isinstance(g, dict) else graph_to_dict(g) for g in graphs]
        self.descs, self._keep = graphs_to_descs(self.graphs)
        self.F = int(F)
        self.n = len(self.graphs)

    def stats(self) -> dict:
        st = np.zeros(7, np.int64)
        rc = self.L.hostemu_stats(self.descs, self.n, self.F, st.ctypes.data)
        if rc:
            raise ValueError(self.L.hostemu_error().decode())
        return dict(zip(("W", "terms", "slow_terms", "columns", "max_term_bytes", "narrow_terms",
                         "hybrid_terms"), st.tolist()))

    def eval(self, gi, params, pairs: bool = False) -> np.ndarray:
        """Complex amplitudes; pairs=True evaluates two rows at a time (the
        two-shots-per-thread path of the kernels)."""
        p = np.ascontiguousarray(params, np.uint8)
        out = np.zeros((p.shape[0], 2))
        rc = self.L.hostemu_eval(self.descs, self.n, self.F, gi,
                                 p.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), p.shape[0],
                                 p.shape[1], 4 if pairs else 0, out.ctypes.data, None)
        assert rc == 0, self.L.hostemu_error()
        return out[:, 0] + 1j * out[:, 1]

    def eval_terms(self, gi, params, pairs: bool = False) -> np.ndarray:
        p = np.ascontiguousarray(params, np.uint8)
        G = int(np.asarray(self.graphs[gi]["pf_phase_idx"]).shape[0])
        out = np.zeros((p.shape[0], G, 5), np.int64)
        rc = self.L.hostemu_eval(self.descs, self.n, self.F, gi,
                                 p.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), p.shape[0],
                                 p.shape[1], 3 if pairs else 2, out.ctypes.data, None)
        assert rc == 0, self.L.hostemu_error()
        return out

    def sample(self, f, seed, mode):
        f = np.ascontiguousarray(f, np.uint8)
        B = f.shape[0]
        out = np.zeros((B, max(self.n - 1, 1)), np.uint8)
        amp = np.zeros((B, self.n))
        rc = self.L.hostemu_sample(self.descs, self.n, self.F,
                                   f.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), B, seed, mode,
                                   out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                                   amp.ctypes.data)
        assert rc == 0, self.L.hostemu_error()
        return out, amp


def canonical_terms(t: np.ndarray) -> np.ndarray:
    """(..., 5) (a,b,c,d,pw): divide by 2 while all four are even and nonzero."""
    t = t.copy()
    for _ in range(130):
        c = t[..., :4]
        red = np.all(c % 2 == 0, axis=-1) & np.any(c != 0, axis=-1)
        if not red.any():
            break
        t[..., :4] = np.where(red[..., None], c // 2, c)
        t[..., 4] = t[..., 4] + red
    zero = ~np.any(t[..., :4] != 0, axis=-1)
    t[..., 4] = np.where(zero, 0, t[..., 4])  # the exponent of 0 is meaningless
    return t
