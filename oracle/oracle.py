"""Python access to the CPU checkers (test infrastructure only).

``PortOracle`` loads ``oracle/libksim_oracle.so`` (the C restatement);
``RefOracle`` loads ``oracle/_ref/libksim_ref.so`` (the reference's own
``zx_eval.hpp`` compiled unmodified, driven by ``oracle/ref_driver.cpp``).
Both take reference-style graph dicts (``sample/sampler.py:21-43`` layout) and
mirror ``kokkos_sim.Component`` (``kokkos_sim.cpp:188-241``, ``:157-185``).

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
legs may import this module.  ``make -C oracle`` builds both libraries.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

from ksim_b200._abi import GraphDesc, graphs_to_descs
from ksim_b200.program import graph_to_dict

HERE = Path(__file__).resolve().parent
PORT_LIB = HERE / "libksim_oracle.so"
REF_LIB = HERE / "_ref" / "libksim_ref.so"

_u8p = ctypes.POINTER(ctypes.c_uint8)
_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)


def build(ref_tree: str | None = None) -> None:
    """Compile the checkers (``oracle/Makefile``)."""
    cmd = ["make", "-s", "-C", str(HERE)]
    if ref_tree:
        cmd.append(f"REF={ref_tree}")
    subprocess.run(cmd, check=True)


def _load(path: Path, prefix: str):
    if not path.exists():
        raise FileNotFoundError(f"{path} not built (run `make -C oracle`)")
    L = ctypes.CDLL(str(path))
    sample = getattr(L, f"{prefix}sample")
    sample.restype = ctypes.c_int
    sample.argtypes = [ctypes.POINTER(GraphDesc), ctypes.c_int, ctypes.c_int, _u8p, ctypes.c_int64,
                       ctypes.c_int64, ctypes.c_uint64, ctypes.c_int, _u8p, _dp, ctypes.c_int]
    ev = getattr(L, f"{prefix}eval")
    ev.restype = ctypes.c_int
    ev.argtypes = [ctypes.POINTER(GraphDesc), ctypes.c_int, ctypes.c_int, _u8p, ctypes.c_int64,
                   ctypes.c_int64, _dp]
    return L


class _Oracle:
    prefix = ""
    path: Path = PORT_LIB
    _cache: dict = {}

    def __init__(self, graphs: list, num_f: int):
        key = (type(self).__name__, str(self.path))
        if key not in _Oracle._cache:
            _Oracle._cache[key] = _load(self.path, self.prefix)
        self.L = _Oracle._cache[key]
        self.graphs = [g if isinstance(g, dict) else graph_to_dict(g) for g in graphs]
        self.descs, self._keep = graphs_to_descs(self.graphs)
        self.num_f = int(num_f)
        self.n_out = len(self.graphs) - 1

    def sample(self, f_sel, seed: int, rng_mode: int = 0, shot_offset: int = 0,
               n_threads: int = 0, return_amp: bool = False):
        f = np.ascontiguousarray(f_sel, dtype=np.uint8)
        B = f.shape[0]
        if f.ndim != 2 or f.shape[1] != self.num_f:
            raise ValueError("f_sel column count != F")
        out = np.zeros((B, max(self.n_out, 1)), np.uint8)
        amp = np.zeros((B, self.n_out + 1), np.float64) if return_amp else None
        rc = getattr(self.L, f"{self.prefix}sample")(
            self.descs, len(self.graphs), self.num_f, f.ctypes.data_as(_u8p), B, shot_offset,
            ctypes.c_uint64(seed & (2**64 - 1)), rng_mode, out.ctypes.data_as(_u8p),
            amp.ctypes.data_as(_dp) if amp is not None else None, n_threads)
        if rc:
            raise RuntimeError(f"oracle sample failed ({rc})")
        return (out, amp) if return_amp else out

    def eval(self, graph: int, params) -> np.ndarray:
        p = np.ascontiguousarray(params, dtype=np.uint8)
        if p.ndim != 2:
            raise ValueError("params must be 2-D")
        B, P = p.shape
        out = np.zeros((B, 2), np.float64)
        rc = getattr(self.L, f"{self.prefix}eval")(
            self.descs, len(self.graphs), graph, p.ctypes.data_as(_u8p), B, P,
            out.ctypes.data_as(_dp))
        if rc:
            raise RuntimeError(f"oracle eval failed ({rc})")
        return out[:, 0] + 1j * out[:, 1]

    def eval_abs(self, graph: int, params) -> np.ndarray:
        a = self.eval(graph, params)
        re, im = a.real, a.imag
        return np.sqrt(re * re + im * im)


class PortOracle(_Oracle):
    """The C restatement (``oracle/ksim_oracle.c``)."""
    prefix = "oracle_"
    path = PORT_LIB

    def eval_terms(self, graph: int, params) -> np.ndarray:
        """(B, G, 5) int64 per-term (a, b, c, d, pw)."""
        p = np.ascontiguousarray(params, dtype=np.uint8)
        B, P = p.shape
        G = int(self.descs[graph].G)
        out = np.zeros((B, G, 5), np.int64)
        f = self.L.oracle_eval_terms
        f.restype = ctypes.c_int
        f.argtypes = [ctypes.POINTER(GraphDesc), ctypes.c_int, ctypes.c_int, _u8p,
                      ctypes.c_int64, ctypes.c_int64, _i64p]
        if f(self.descs, len(self.graphs), graph, p.ctypes.data_as(_u8p), B, P,
             out.ctypes.data_as(_i64p)):
            raise RuntimeError("oracle eval_terms failed")
        return out


class RefOracle(_Oracle):
    """The reference's own zx_eval.hpp (``oracle/_ref``)."""
    prefix = "oracle_ref_"
    path = REF_LIB

    @staticmethod
    def available() -> bool:
        return REF_LIB.exists()


def _port_lib():
    return _Oracle._cache.setdefault(("PortOracle", str(PORT_LIB)), _load(PORT_LIB, "oracle_"))


def philox4x32_10(ctr, key) -> tuple:
    """Philox4x32-10 block: ctr (4 x u32), key (2 x u32) -> 4 x u32."""
    L = _port_lib()
    f = L.oracle_philox4x32_10
    f.restype = None
    c = (ctypes.c_uint32 * 4)(*[int(x) & 0xFFFFFFFF for x in ctr])
    k = (ctypes.c_uint32 * 2)(*[int(x) & 0xFFFFFFFF for x in key])
    o = (ctypes.c_uint32 * 4)()
    f(c, k, o)
    return tuple(int(x) for x in o)


def philox_uniform(seed: int, shot: int, output: int) -> float:
    L = _port_lib()
    f = L.oracle_philox_uniform
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32]
    return float(f(seed, shot, output))


def exp2_int(n: int) -> float:
    L = _port_lib()
    f = L.oracle_exp2_int
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.c_int64]
    return float(f(n))


def max_threads() -> int:
    L = _port_lib()
    return int(L.oracle_max_threads())


def program_sample(prog, f_params, seed: int, rng_mode: int = 0, oracle_cls=PortOracle,
                   n_threads: int = 0, shot_offset: int = 0):
    """KokkosProgramSampler.sample semantics (sampler.py:57-67) on an oracle."""
    B = f_params.shape[0]
    outs = []
    for k, comp in enumerate(prog.components):
        F = int(np.asarray(comp.f_selection).shape[0])
        oc = oracle_cls(comp.graphs, F)
        f_sel = np.ascontiguousarray(f_params[:, np.asarray(comp.f_selection, np.int64)],
                                     dtype=np.uint8)
        outs.append(oc.sample(f_sel, (seed + 0x9E37 * k) & (2**64 - 1), rng_mode,
                              shot_offset=shot_offset, n_threads=n_threads)
                    [:, :len(comp.graphs) - 1])
    combined = np.concatenate(outs, axis=1) if outs else np.zeros((B, 0), np.uint8)
    return combined[:, np.argsort(prog.output_order)]


def noise_sample(channel_probs, error_transform, B: int, shot_offset: int, seed: int) -> np.ndarray:
    """The device noise draw restated on the CPU (``oracle_noise_sample``):
    (B, num_f) uint8 for shots shot_offset .. shot_offset + B - 1."""
    L = _port_lib()
    f = L.oracle_noise_sample
    f.restype = ctypes.c_int
    f.argtypes = [_dp, ctypes.POINTER(ctypes.c_int32), ctypes.c_int, _u8p, ctypes.c_int, ctypes.c_int,
                  ctypes.c_int64, ctypes.c_int64, ctypes.c_uint64, _u8p]
    probs = [np.asarray(p, np.float64).reshape(-1) for p in channel_probs]
    flat = np.ascontiguousarray(np.concatenate(probs) if probs else np.zeros(1))
    n_bits = np.ascontiguousarray([int(round(np.log2(len(p)))) for p in probs] or [0], np.int32)
    T = np.ascontiguousarray(np.asarray(error_transform, np.uint8))
    out = np.zeros((B, T.shape[0]), np.uint8)
    rc = f(flat.ctypes.data_as(_dp), n_bits.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(probs),
           T.ctypes.data_as(_u8p), T.shape[0], T.shape[1], B, shot_offset, seed & (2**64 - 1),
           out.ctypes.data_as(_u8p))
    if rc:
        raise RuntimeError("oracle noise sample failed")
    return out
