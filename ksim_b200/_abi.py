"""ctypes view of the C ABI declared in ``include/ksim_b200.h``.

The library is ``ksim_b200/lib/libksim_b200.so`` (built in-tree by
``ksim_b200/build.py``).  There is no fallback: if it is missing or a CUDA
device is absent, the calls raise.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

LIB_DIR = Path(__file__).resolve().parent / "lib"
LIB_PATH = LIB_DIR / "libksim_b200.so"

KSIM_OK = 0
KSIM_ERR_INVALID_ARGUMENT = 1
KSIM_ERR_MALFORMED_PROGRAM = 2
KSIM_ERR_CUDA = 3
KSIM_ERR_OUT_OF_MEMORY = 4
KSIM_ERR_TIMEOUT = 5
KSIM_ERR_UNSUPPORTED = 6
KSIM_ERR_NOT_FOUND = 7
KSIM_ERR_CANCELLED = 8
KSIM_ERR_NO_DEVICE = 9
KSIM_ERR_INTERNAL = 10

RNG_XORSHIFT = 0
RNG_PHILOX = 1

FLAG_INT64_RISK = 1
FLAG_PREV_NONPOSITIVE = 2
FLAG_NAN = 4
FLAG_WAIT_TIMEOUT = 8

_u8p = ctypes.POINTER(ctypes.c_uint8)
_i32p = ctypes.POINTER(ctypes.c_int32)
_f32p = ctypes.POINTER(ctypes.c_float)


class GraphDesc(ctypes.Structure):
    """``ksim_graph_desc``: one FlatScalarGraph as 19 borrowed arrays."""
    _fields_ = [
        ("G", ctypes.c_int32), ("P", ctypes.c_int32), ("Tnp", ctypes.c_int32),
        ("Thp", ctypes.c_int32), ("Tpp", ctypes.c_int32), ("Tph", ctypes.c_int32),
        ("np_phases", _u8p), ("np_params", _u8p), ("np_counts", _i32p),
        ("hp_coeffs", _u8p), ("hp_params", _u8p),
        ("pp_psi_c", _u8p), ("pp_psi_p", _u8p), ("pp_phi_c", _u8p), ("pp_phi_p", _u8p),
        ("ph_alpha", _u8p), ("ph_alpha_p", _u8p), ("ph_beta", _u8p), ("ph_beta_p", _u8p),
        ("ph_counts", _i32p),
        ("pf_phase_idx", _u8p), ("pf_floatfactor", _i32p), ("pf_power2", _i32p),
        ("pf_approx_f32", _f32p), ("pf_has_approx", ctypes.c_int32),
    ]


class BatchJob(ctypes.Structure):
    """``ksim_batch_job``."""
    _fields_ = [
        ("comp", ctypes.c_void_p), ("d_f", ctypes.c_void_p), ("f_stride", ctypes.c_int64),
        ("d_f_sel", ctypes.c_void_p), ("d_out", ctypes.c_void_p), ("out_stride", ctypes.c_int64),
        ("out_col0", ctypes.c_int64), ("d_out_cols", ctypes.c_void_p), ("B", ctypes.c_int64),
        ("shot_offset", ctypes.c_int64), ("seed", ctypes.c_uint64), ("rng_mode", ctypes.c_int32),
    ]


class BatchTuning(ctypes.Structure):
    """``ksim_batch_tuning``."""
    _fields_ = [("threads", ctypes.c_int32), ("slot_bytes", ctypes.c_int32),
                ("ctas_per_sm", ctypes.c_int32), ("use_graph", ctypes.c_int32)]


class ServerConfig(ctypes.Structure):
    """``ksim_server_config``."""
    _fields_ = [("device", ctypes.c_int32), ("arena_bytes", ctypes.c_int64),
                ("max_requests", ctypes.c_int32), ("max_jobs", ctypes.c_int32),
                ("threads", ctypes.c_int32), ("slot_bytes", ctypes.c_int32),
                ("ctas_per_sm", ctypes.c_int32), ("idle_us", ctypes.c_int32)]


class ServerStats(ctypes.Structure):
    """``ksim_server_stats``."""
    _fields_ = [(n, ctypes.c_int64) for n in (
        "submitted", "completed", "failed", "cancelled", "shots_completed", "loop_launches",
        "side_launches", "pending", "in_flight", "arena_in_use", "arena_capacity")]


_U8_KEYS = ("np_phases", "np_params", "hp_coeffs", "hp_params", "pp_psi_c", "pp_psi_p",
            "pp_phi_c", "pp_phi_p", "ph_alpha", "ph_alpha_p", "ph_beta", "ph_beta_p",
            "pf_phase_idx")
_I32_KEYS = ("np_counts", "ph_counts", "pf_floatfactor", "pf_power2")


def _dim(a: np.ndarray, d: int) -> int:
    # kokkos_sim.cpp:93-96: a missing dimension reads as 1
    return int(a.shape[d]) if d < a.ndim else 1


def graphs_to_descs(graphs: list) -> tuple:
    """Build a ``GraphDesc[n]`` array from reference-style graph dicts.

    Returns ``(descs, keepalive)``; ``keepalive`` holds the contiguous arrays
    the pointers refer to and must live as long as ``descs`` is used.
    """
    n = len(graphs)
    descs = (GraphDesc * max(n, 1))()
    keep = []
    for k, g in enumerate(graphs):
        d = descs[k]
        arrs = {}
        for key in _U8_KEYS:
            arrs[key] = np.ascontiguousarray(g[key], dtype=np.uint8)
        for key in _I32_KEYS:
            arrs[key] = np.ascontiguousarray(g[key], dtype=np.int32)
        apx = g.get("pf_approx_f32")
        if apx is None:
            apx = np.asarray(g["pf_approx"], np.complex64).view(np.float32)
        arrs["pf_approx_f32"] = np.ascontiguousarray(apx, dtype=np.float32)
        d.G = _dim(arrs["pf_phase_idx"], 0)
        d.P = _dim(arrs["np_params"], 2)
        d.Tnp = _dim(arrs["np_phases"], 1)
        d.Thp = _dim(arrs["hp_coeffs"], 1)
        d.Tpp = _dim(arrs["pp_psi_c"], 1)
        d.Tph = _dim(arrs["ph_alpha"], 1)
        for key in _U8_KEYS:
            setattr(d, key, arrs[key].ctypes.data_as(_u8p))
        for key in _I32_KEYS:
            setattr(d, key, arrs[key].ctypes.data_as(_i32p))
        d.pf_approx_f32 = arrs["pf_approx_f32"].ctypes.data_as(_f32p)
        d.pf_has_approx = 1 if bool(g["pf_has_approx"]) else 0
        keep.append(arrs)
    return descs, keep


def graph_shapes_ok(graphs: list) -> None:
    """Raise ValueError when a graph's arrays disagree with its own G/P/T*.

    The reference reads such programs out of bounds; here they are rejected
    before upload (the native side re-checks what it can see)."""
    for k, g in enumerate(graphs):
        G = _dim(np.asarray(g["pf_phase_idx"]), 0)
        P = _dim(np.asarray(g["np_params"]), 2)
        fams = (("np_phases", "np_params"), ("hp_coeffs", "hp_params"),
                ("pp_psi_c", "pp_psi_p"), ("pp_phi_c", "pp_phi_p"),
                ("ph_alpha", "ph_alpha_p"), ("ph_beta", "ph_beta_p"))
        for ck, pk in fams:
            c = np.asarray(g[ck])
            p = np.asarray(g[pk])
            T = _dim(c, 1)
            if c.size != G * T or p.size != G * T * P:
                raise ValueError(
                    f"graph {k}: {ck}/{pk} sizes {c.size}/{p.size} do not match "
                    f"G={G}, T={T}, P={P}")
        for key, want in (("np_counts", G), ("ph_counts", G), ("pf_power2", G),
                          ("pf_floatfactor", 4 * G)):
            if np.asarray(g[key]).size != want:
                raise ValueError(f"graph {k}: {key} has {np.asarray(g[key]).size} values, "
                                 f"expected {want}")


_lib = None


def lib() -> ctypes.CDLL:
    """Load ``libksim_b200.so`` once; raise loudly if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("KSIM_B200_LIB", str(LIB_PATH)))
    if not path.exists():
        raise ImportError(
            f"{path} is missing: build it with `python -m ksim_b200.build` "
            "(nvcc, sm_100a). There is no CPU fallback.")
    L = ctypes.CDLL(str(path))
    _declare(L)
    _lib = L
    return L


def _declare(L: ctypes.CDLL) -> None:
    vp = ctypes.c_void_p
    i32, i64, u64, u32 = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_uint32
    dp = ctypes.POINTER(ctypes.c_double)
    i64p = ctypes.POINTER(ctypes.c_int64)
    sigs = {
        "ksim_last_error": (ctypes.c_char_p, []),
        "ksim_abi_version": (i32, []),
        "ksim_device_count": (i32, []),
        "ksim_component_create": (i32, [ctypes.POINTER(GraphDesc), i32, i32, i32,
                                        ctypes.POINTER(vp)]),
        "ksim_component_destroy": (None, [vp]),
        "ksim_component_n_out": (i32, [vp]),
        "ksim_component_num_f": (i32, [vp]),
        "ksim_component_n_graphs": (i32, [vp]),
        "ksim_component_words": (i32, [vp]),
        "ksim_component_image_bytes": (i64, [vp]),
        "ksim_component_sample": (i32, [vp, _u8p, i64, u64, i32, _u8p]),
        "ksim_component_sample_device": (i32, [vp, vp, i64, i64, u64, i32, vp, i64, i64,
                                               vp, vp]),
        "ksim_component_sample_device_noalloc": (i32, [vp, vp, i64, i64, u64, i32, vp, i64,
                                                       i64, vp, vp]),
        "ksim_component_eval_abs": (i32, [vp, i32, _u8p, i64, i64, dp]),
        "ksim_component_eval": (i32, [vp, i32, _u8p, i64, i64, dp]),
        "ksim_component_eval_terms": (i32, [vp, i32, _u8p, i64, i64, i64p]),
        "ksim_component_status": (i32, [vp, ctypes.POINTER(u32), i32]),
        "ksim_component_set_launch": (i32, [vp, i32, i32, i32]),
        "ksim_component_set_wait_limit": (i32, [vp, i64]),
        "ksim_component_get_launch": (i32, [vp, ctypes.POINTER(i32), ctypes.POINTER(i32),
                                            ctypes.POINTER(i32)]),
        "ksim_component_stats": (i32, [vp, i64p, i64p, i64p, i64p]),
        "ksim_program_create": (i32, [ctypes.POINTER(vp), i32, ctypes.POINTER(_i32p), _i32p,
                                      _i32p, i32, ctypes.POINTER(vp)]),
        "ksim_program_destroy": (None, [vp]),
        "ksim_program_n_outputs": (i32, [vp]),
        "ksim_program_min_f_cols": (i32, [vp]),
        "ksim_program_sample": (i32, [vp, _u8p, i64, i64, u64, i32, _u8p]),
        "ksim_program_sample_device": (i32, [vp, vp, i64, i64, i64, u64, i32, vp, vp]),
        "ksim_program_sample_packed": (i32, [vp, _u8p, i64, i64, u64, i32, _u8p]),
        "ksim_measure_int_peak": (i32, [i32, dp, dp]),
        "ksim_measure_alu_peak": (i32, [i32, dp, dp]),
        "ksim_work_model": (i32, [ctypes.POINTER(GraphDesc), i32, i32, dp, i64p]),
        "ksim_batch_create": (i32, [ctypes.POINTER(BatchJob), i32, ctypes.POINTER(BatchTuning),
                                    ctypes.POINTER(vp)]),
        "ksim_batch_set_seeds": (i32, [vp, ctypes.POINTER(u64)]),
        "ksim_program_job": (i32, [vp, i32, vp, i64, vp, i64, i64, u64, i32,
                                   ctypes.POINTER(BatchJob)]),
        "ksim_program_n_components": (i32, [vp]),
        "ksim_batch_launch": (i32, [vp, vp]),
        "ksim_batch_info": (i32, [vp, i64p, ctypes.POINTER(i32), ctypes.POINTER(i32)]),
        "ksim_batch_destroy": (None, [vp]),
        "ksim_noise_create": (i32, [dp, ctypes.POINTER(i32), i32, _u8p, i32, i32, i32,
                                    ctypes.POINTER(vp)]),
        "ksim_noise_destroy": (None, [vp]),
        "ksim_noise_num_f": (i32, [vp]),
        "ksim_noise_num_channels": (i32, [vp]),
        "ksim_noise_sample_device": (i32, [vp, i64, i64, u64, vp, i64, vp]),
        "ksim_noise_sample": (i32, [vp, i64, i64, u64, _u8p]),
        "ksim_program_sample_noisy": (i32, [vp, vp, i64, u64, u64, i32, _u8p]),
        "ksim_server_create": (i32, [ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]),
        "ksim_server_submit": (i32, [vp, vp, vp, i64, i64, i64, u64, i32, vp, i64p]),
        "ksim_server_wait": (i32, [vp, i64, i32, dp, dp]),
        "ksim_server_poll": (i32, [vp, i64, ctypes.POINTER(i32)]),
        "ksim_server_cancel": (i32, [vp, i64]),
        "ksim_server_get_stats": (i32, [vp, ctypes.POINTER(ServerStats)]),
        "ksim_server_destroy": (None, [vp]),
    }
    for name, (res, args) in sigs.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


class KsimError(RuntimeError):
    """A native call failed with a status other than invalid-argument."""

    def __init__(self, status: int, message: str):
        super().__init__(f"ksim_b200 error {status}: {message}")
        self.status = status


def status_error(status: int, msg: str) -> Exception:
    """The exception a non-OK ``ksim_status`` maps to (ValueError for bad
    arguments, as the reference's std::invalid_argument surfaces)."""
    if status in (KSIM_ERR_INVALID_ARGUMENT, KSIM_ERR_MALFORMED_PROGRAM):
        return ValueError(msg)
    if status == KSIM_ERR_OUT_OF_MEMORY:
        return MemoryError(msg)
    if status == KSIM_ERR_TIMEOUT:
        return TimeoutError(msg)
    return KsimError(status, msg)


def check(status: int) -> None:
    """Raise the exception of a failing ``ksim_status`` with the library's
    message of the last failing call on this thread."""
    if status == KSIM_OK:
        return
    raise status_error(status, (lib().ksim_last_error() or b"").decode(errors="replace"))


def u8ptr(a: np.ndarray):
    return a.ctypes.data_as(_u8p)


def i32ptr(a: np.ndarray):
    return a.ctypes.data_as(_i32p)
