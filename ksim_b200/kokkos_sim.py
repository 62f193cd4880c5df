"""Drop-in for the reference's native module ``kokkos_sim``.

Same class, constructor, methods and errors as the nanobind module of
``src/cpp/ksim/kokkos_sim.cpp:244-252``::

    Component(graphs: list[dict], num_f: int)
    Component.sample(f_sel: uint8 (B, num_f), seed: uint64) -> uint8 (B, max(n_out, 1))
    Component.eval_abs(graph: int, params: uint8 (B, P)) -> float64 (B,)
    Component.n_out

backed by ``libksim_b200.so`` (sm_100a kernels behind the C ABI in
``include/ksim_b200.h``).  ``sample`` is bit-identical to kokkos_sim for the
same seed (its xorshift stream); ``rng_mode=RNG_PHILOX`` selects the
counter-based Philox4x32-10 stream instead.  Extras beyond the reference:
``eval`` (complex amplitude), ``eval_terms`` (exact per-term numerators),
``status`` (advisory kernel flags), ``set_launch`` (launch shape).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import RNG_PHILOX, RNG_XORSHIFT, check, lib
from .program import graph_to_dict

__all__ = ["Component", "RNG_XORSHIFT", "RNG_PHILOX"]

_U64 = 2**64


def _as_u64(seed) -> int:
    # nanobind's uint64_t caster rejects negatives and values >= 2**64 with TypeError
    if isinstance(seed, bool) or not isinstance(seed, (int, np.integer)):
        raise TypeError(f"seed must be an integer, got {type(seed).__name__}")
    s = int(seed)
    if s < 0 or s >= _U64:
        raise TypeError(f"seed {s} does not fit in uint64")
    return s


def _rows_u8(a, name: str) -> np.ndarray:
    arr = np.ascontiguousarray(a, dtype=np.uint8)
    if arr.ndim != 2:
        raise TypeError(f"{name} must be a 2-D uint8 array, got {arr.ndim}-D")
    return arr


class Component:
    """One FlatComponent uploaded to the GPU (``KokkosTsimComponent``)."""

    def __init__(self, graphs: list, num_f: int, device: int = -1):
        L = lib()
        # reference-style dicts (sampler.py:21-43 layout) or FlatScalarGraph objects
        graphs = [g if isinstance(g, dict) else graph_to_dict(g) for g in graphs]
        _abi.graph_shapes_ok(graphs)
        descs, keep = _abi.graphs_to_descs(graphs)
        h = ctypes.c_void_p()
        check(L.ksim_component_create(descs, len(graphs), int(num_f), int(device), ctypes.byref(h)))
        del keep
        self._h = h
        self._L = L
        self._num_f = int(num_f)
        self._n_out = int(L.ksim_component_n_out(h))
        self._graph_sizes = [int(np.asarray(g["pf_phase_idx"]).shape[0]) for g in graphs]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.ksim_component_destroy(h)
            self._h = None

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    @property
    def n_out(self) -> int:
        return self._n_out

    @property
    def num_f(self) -> int:
        return self._num_f

    @property
    def words(self) -> int:
        """64-bit words per parameter vector in the device image."""
        return int(self._L.ksim_component_words(self._h))

    def sample(self, f_sel, seed, rng_mode: int = RNG_XORSHIFT) -> np.ndarray:
        f = _rows_u8(f_sel, "f_sel")
        if f.shape[1] != self._num_f:
            raise ValueError("f_sel column count != F")
        s = _as_u64(seed)
        B = f.shape[0]
        out = np.zeros((B, max(self._n_out, 1)), np.uint8)
        check(self._L.ksim_component_sample(self._h, _abi.u8ptr(f), B, s, int(rng_mode),
                                            _abi.u8ptr(out)))
        return out

    def _params(self, graph: int, params):
        p = _rows_u8(params, "params")
        if not 0 <= int(graph) < len(self._graph_sizes):
            raise IndexError(f"graph {graph} out of range")
        return p

    def eval_abs(self, graph: int, params) -> np.ndarray:
        p = self._params(graph, params)
        out = np.zeros(p.shape[0], np.float64)
        check(self._L.ksim_component_eval_abs(self._h, int(graph), _abi.u8ptr(p), p.shape[0],
                                              p.shape[1],
                                              out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def eval(self, graph: int, params) -> np.ndarray:
        """Complex amplitude of ``graph`` for explicit parameter rows."""
        p = self._params(graph, params)
        out = np.zeros((p.shape[0], 2), np.float64)
        check(self._L.ksim_component_eval(self._h, int(graph), _abi.u8ptr(p), p.shape[0],
                                          p.shape[1],
                                          out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out[:, 0] + 1j * out[:, 1]

    def eval_terms(self, graph: int, params) -> np.ndarray:
        """(B, G, 5) int64: each term's exact (a, b, c, d, pw)."""
        p = self._params(graph, params)
        G = self._graph_sizes[int(graph)]
        out = np.zeros((p.shape[0], G, 5), np.int64)
        check(self._L.ksim_component_eval_terms(self._h, int(graph), _abi.u8ptr(p), p.shape[0],
                                                p.shape[1],
                                                out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        return out

    def status(self, reset: bool = False) -> int:
        """OR of KSIM_FLAG_* raised by this component's kernels."""
        f = ctypes.c_uint32()
        check(self._L.ksim_component_status(self._h, ctypes.byref(f), 1 if reset else 0))
        return int(f.value)

    def set_launch(self, threads: int = 0, staged: int = -1, slot_bytes: int = 0) -> None:
        check(self._L.ksim_component_set_launch(self._h, int(threads), int(staged), int(slot_bytes)))

    def set_wait_limit(self, polls: int = 0) -> None:
        """Bound of the staging waits of this component's kernels in mbarrier
        polls (0: the built-in bound).  A wait that runs out makes the host
        calls raise TimeoutError (KSIM_ERR_TIMEOUT)."""
        check(self._L.ksim_component_set_wait_limit(self._h, int(polls)))

    def get_launch(self) -> dict:
        t, s, b = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        check(self._L.ksim_component_get_launch(self._h, ctypes.byref(t), ctypes.byref(s),
                                                ctypes.byref(b)))
        return {"threads": t.value, "staged": s.value, "slot_bytes": b.value}

    def stats(self) -> dict:
        a, b, c, d = (ctypes.c_int64() for _ in range(4))
        check(self._L.ksim_component_stats(self._h, ctypes.byref(a), ctypes.byref(b),
                                           ctypes.byref(c), ctypes.byref(d)))
        return {"terms": a.value, "slow_terms": b.value, "columns": c.value,
                "max_term_bytes": d.value,
                "image_bytes": int(self._L.ksim_component_image_bytes(self._h)),
                "words": self.words}
