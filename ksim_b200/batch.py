"""Batched sampling: many FlatPrograms in one graph-captured launch.

``BatchSampler(programs, shots)`` uploads every program once, keeps one device
input buffer (the full f matrix) and one device output buffer per program,
and turns every component of every program into a job of one
``ksim_batch`` (``include/ksim_b200.h``): longest-first work items pulled by
persistent CTAs, one kernel per (W, term paths) class of jobs, the class
kernels chained on one stream as programmatic dependent launches (each
starts while the one before it drains), all captured in a CUDA graph and
replayed.  Each
program's result is bit-identical to ``B200ProgramSampler(prog).sample``
with the same seed — shot s of a job always uses stream index s, whatever
else shares the launch.

``tune()`` is the autotuner: it times a small grid of launch shapes (shots
per work item, staging slot size, persistent CTAs per SM) on the batch
itself and keeps the fastest; results are cached per GPU and batch shape in
``$KSIM_B200_TUNE_CACHE`` (default ``~/.cache/ksim_b200/tuning.json``).
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os
from pathlib import Path

import numpy as np

from . import _abi
from ._abi import RNG_XORSHIFT, check, lib
from .kokkos_sim import _as_u64
from .sampler import B200ProgramSampler

__all__ = ["BatchSampler", "tune_cache_path"]

_DEFAULT_TUNING = {"threads": 128, "slot_bytes": 14336, "ctas_per_sm": 0}
_CANDIDATES = [
    {"threads": t, "slot_bytes": s, "ctas_per_sm": c}
    for t in (64, 128, 256) for s in (8192, 12288, 14336, 16384) for c in (0, 4)
]


def tune_cache_path() -> Path:
    p = os.environ.get("KSIM_B200_TUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "ksim_b200" / "tuning.json"


def _load_cache() -> dict:
    try:
        return json.loads(tune_cache_path().read_text())
    except (OSError, ValueError):
        return {}


def _store_cache(key: str, value: dict) -> None:
    path = tune_cache_path()
    cache = _load_cache()
    cache[key] = value
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        tmp = path.with_suffix(".tmp")
        tmp.write_text(json.dumps(cache, indent=1, sort_keys=True))
        tmp.replace(path)
    except OSError:
        pass


class BatchSampler:
    """Sample several FlatPrograms in one graph launch.

    ``programs``: list of FlatProgram; ``shots``: shots per program.
    Inputs come from host arrays (``set_inputs``) or stay on the device
    (``device_inputs``); outputs are read with ``results``.
    """

    def __init__(self, programs, shots, seeds=None, rng_mode: int = RNG_XORSHIFT,
                 device: int = 0, tuning: dict | None = None, use_graph: bool = True,
                 n_f=None):
        import torch
        self._torch = torch
        self.L = lib()
        self.device = int(device)
        self.dev = torch.device("cuda", self.device)
        self.programs = list(programs)
        self.shots = [int(b) for b in shots]
        if len(self.shots) != len(self.programs):
            raise ValueError("one shot count per program")
        self.rng_mode = int(rng_mode)
        self.seeds = [int(s) for s in (seeds if seeds is not None else range(len(self.programs)))]
        self.samplers = [B200ProgramSampler(p, device=self.device) for p in self.programs]
        # width of each program's f matrix (at least max(f_selection) + 1)
        self.n_f = [max(s.min_f_cols, int(n_f[i]) if n_f is not None else 0)
                    for i, s in enumerate(self.samplers)]
        self.d_f = [torch.zeros((b, nf), dtype=torch.uint8, device=self.dev)
                    for b, nf in zip(self.shots, self.n_f)]
        self.d_out = [torch.zeros((b, s.num_outputs), dtype=torch.uint8, device=self.dev)
                      for b, s in zip(self.shots, self.samplers)]
        self.use_graph = bool(use_graph)
        self._h = None
        self.tuning = dict(tuning or _DEFAULT_TUNING)
        self._build(self.tuning)

    # -- construction -------------------------------------------------------
    def _jobs(self):
        jobs = []
        for pi, (s, b) in enumerate(zip(self.samplers, self.shots)):
            seed = _as_u64(self.seeds[pi])
            n_c = int(self.L.ksim_program_n_components(s.handle))
            for k in range(n_c):
                j = _abi.BatchJob()
                check(self.L.ksim_program_job(
                    s.handle, k, ctypes.c_void_p(self.d_f[pi].data_ptr()), max(self.n_f[pi], 0),
                    ctypes.c_void_p(self.d_out[pi].data_ptr()), b, 0, seed, self.rng_mode,
                    ctypes.byref(j)))
                jobs.append(j)
        return jobs

    def _build(self, tuning: dict) -> None:
        self._destroy()
        jobs = self._jobs()
        self._n_jobs = len(jobs)
        arr = (_abi.BatchJob * max(len(jobs), 1))(*jobs)
        t = _abi.BatchTuning(int(tuning.get("threads", 128)), int(tuning.get("slot_bytes", 16384)),
                             int(tuning.get("ctas_per_sm", 0)), 1 if self.use_graph else 0)
        h = ctypes.c_void_p()
        check(self.L.ksim_batch_create(arr, len(jobs), ctypes.byref(t), ctypes.byref(h)))
        self._h = h
        self.tuning = dict(tuning)

    def _destroy(self) -> None:
        if self._h is not None and self._h.value:
            self.L.ksim_batch_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self._destroy()
        except Exception:
            pass

    # -- use ----------------------------------------------------------------
    @property
    def total_shots(self) -> int:
        return int(sum(self.shots))

    def info(self) -> dict:
        n, g, l = ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int32()
        check(self.L.ksim_batch_info(self._h, ctypes.byref(n), ctypes.byref(g), ctypes.byref(l)))
        return {"items": n.value, "grid": g.value, "launches": l.value, "jobs": self._n_jobs,
                **self.tuning}

    def set_inputs(self, f_list) -> None:
        """Copy each program's (shots, n_f) uint8 noise matrix to the device."""
        for pi, f in enumerate(f_list):
            f = np.ascontiguousarray(f, dtype=np.uint8)
            if f.shape != (self.shots[pi], self.n_f[pi]):
                raise ValueError(f"program {pi}: f has shape {f.shape}, expected "
                                 f"{(self.shots[pi], self.n_f[pi])}")
            if f.size:
                self.d_f[pi].copy_(self._torch.from_numpy(f), non_blocking=False)

    def set_seeds(self, seeds) -> None:
        self.seeds = [int(s) for s in seeds]
        per_job = []
        for pi, s in enumerate(self.samplers):
            n_c = int(self.L.ksim_program_n_components(s.handle))
            per_job += [(_as_u64(self.seeds[pi]) + 0x9E37 * k) & (2**64 - 1) for k in range(n_c)]
        arr = (ctypes.c_uint64 * len(per_job))(*per_job)
        check(self.L.ksim_batch_set_seeds(self._h, arr))

    def launch(self, stream=None) -> None:
        """Enqueue the whole batch (graph replay) on `stream` (torch stream or None)."""
        st = stream if stream is not None else self._torch.cuda.current_stream(self.dev)
        check(self.L.ksim_batch_launch(self._h, ctypes.c_void_p(st.cuda_stream)))

    def results(self) -> list:
        self._torch.cuda.synchronize(self.dev)
        return [o.cpu().numpy() for o in self.d_out]

    def sample(self, f_list, seeds=None) -> list:
        """Host inputs in, host outputs out (one array per program)."""
        if seeds is not None:
            self.set_seeds(seeds)
        self.set_inputs(f_list)
        self.launch()
        return self.results()

    # -- the plain comparison -----------------------------------------------
    def launch_plain(self, stream=None) -> None:
        """The same work as one program-per-launch calls (the plain GPU path)."""
        st = stream if stream is not None else self._torch.cuda.current_stream(self.dev)
        for pi, s in enumerate(self.samplers):
            if self.shots[pi] == 0:
                continue
            check(self.L.ksim_program_sample_device(
                s.handle, ctypes.c_void_p(self.d_f[pi].data_ptr()), self.shots[pi], self.n_f[pi], 0,
                _as_u64(self.seeds[pi]), self.rng_mode, ctypes.c_void_p(self.d_out[pi].data_ptr()),
                ctypes.c_void_p(st.cuda_stream)))

    # -- autotuner ----------------------------------------------------------
    def signature(self) -> str:
        h = hashlib.sha1()
        for s, b in zip(self.samplers, self.shots):
            for _, kc in s.components:
                st = kc.stats()
                h.update(f"{st['terms']},{st['columns']},{st['words']},{st['max_term_bytes']},"
                         f"{kc.n_out},{b};".encode())
        name = self._torch.cuda.get_device_name(self.dev)
        return f"{name}|{h.hexdigest()}"

    def time_launch(self, reps: int = 3) -> float:
        """Mean ms of one batch launch (CUDA events on the launching stream)."""
        torch = self._torch
        st = torch.cuda.current_stream(self.dev)
        self.launch(st)
        torch.cuda.synchronize(self.dev)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(st)
        for _ in range(reps):
            self.launch(st)
        b.record(st)
        torch.cuda.synchronize(self.dev)
        return a.elapsed_time(b) / reps

    def tune(self, candidates=None, reps: int = 2, use_cache: bool = True) -> dict:
        key = self.signature()
        if use_cache:
            hit = _load_cache().get(key)
            if hit:
                self._build(hit["tuning"])
                return hit
        max_term = max(kc.stats()["max_term_bytes"] for s in self.samplers for _, kc in s.components)
        results = []
        for cand in (candidates or _CANDIDATES):
            if cand["slot_bytes"] < max_term:
                continue
            try:
                self._build(cand)
            except ValueError:
                continue
            results.append((self.time_launch(reps), cand))
        if not results:
            self._build(_DEFAULT_TUNING)
            return {"tuning": dict(_DEFAULT_TUNING), "ms": None}
        ms, best = min(results, key=lambda r: r[0])
        self._build(best)
        rec = {"tuning": dict(best), "ms": ms,
               "tried": [{"ms": m, **c} for m, c in sorted(results, key=lambda r: r[0])]}
        _store_cache(key, rec)
        return rec
