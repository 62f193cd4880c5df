"""Continuous-batching sample server over ``ksim_server`` (``include/ksim_b200.h``).

``Server`` keeps uploaded programs cached on the GPU and serves sample
requests for any of them through one device-resident request loop::

    srv = Server(device=0)
    req = srv.submit(prog, f, seed)        # returns at once
    bits = req.result()                    # (B, num_outputs) uint8, as
                                           # B200ProgramSampler(prog).sample(f, seed)

* Admission: the native scheduler admits requests in arrival order once
  their HBM footprint (f rows + output rows) fits the server's arena and a
  slot is free; admitted requests' tiles are drained by a persistent kernel,
  so requests that arrive while others run are batched into the running work.
* Program cache: ``ProgramCache`` holds uploaded programs keyed by a content
  digest, evicting the least recently used ones when their device images
  exceed ``cache_bytes``; programs with requests in flight are never evicted.
* Results depend only on (program, f, seed, rng_mode): a request returns the
  same bits alone or in any mix.

No reference counterpart: the reference samples one synchronous call at a
time (``kokkos_sim.cpp:188-241``, ``sample/sampler.py:57-67``).
"""
from __future__ import annotations

import ctypes
import hashlib
import threading
import weakref
from collections import OrderedDict

import numpy as np

from . import _abi
from ._abi import RNG_XORSHIFT, check, lib
from .kokkos_sim import _as_u64
from .sampler import B200ProgramSampler

__all__ = ["ProgramCache", "Request", "Server", "program_digest"]


def program_digest(prog) -> str:
    """Content digest of a FlatProgram (every array of every graph, the
    f selections and the output order)."""
    h = hashlib.sha1()
    for comp in prog.components:
        h.update(np.ascontiguousarray(np.asarray(comp.f_selection), np.int32).tobytes())
        h.update(np.ascontiguousarray(np.asarray(comp.output_indices), np.int64).tobytes())
        for g in comp.graphs:
            for name in ("np_phases", "np_params", "np_counts", "hp_coeffs", "hp_params",
                         "pp_psi_c", "pp_psi_p", "pp_phi_c", "pp_phi_p", "ph_alpha",
                         "ph_alpha_p", "ph_beta", "ph_beta_p", "ph_counts", "pf_phase_idx",
                         "pf_floatfactor", "pf_power2", "pf_approx"):
                a = np.ascontiguousarray(np.asarray(getattr(g, name)))
                h.update(f"{name}{a.dtype.str}{a.shape}".encode())
                h.update(a.tobytes())
            h.update(b"apx1" if bool(g.pf_has_approx) else b"apx0")
        h.update(b"|")
    h.update(np.ascontiguousarray(np.asarray(prog.output_order), np.int64).tobytes())
    return h.hexdigest()


class ProgramCache:
    """Uploaded programs by content digest, LRU within ``cache_bytes`` of
    device images; entries with requests in flight are pinned."""

    def __init__(self, device: int, cache_bytes: int = 8 << 30):
        self.device = int(device)
        self.cache_bytes = int(cache_bytes)
        self._entries: OrderedDict = OrderedDict()  # digest -> [sampler, bytes, pins]
        self._ids: dict = {}  # id(prog) -> (weakref, digest)
        self._lock = threading.Lock()
        self.hits = self.misses = self.evictions = 0

    def _digest(self, prog) -> str:
        hit = self._ids.get(id(prog))
        if hit is not None and hit[0]() is prog:
            return hit[1]
        d = program_digest(prog)
        try:
            self._ids[id(prog)] = (weakref.ref(prog), d)
        except TypeError:
            pass
        return d

    @property
    def bytes(self) -> int:
        return sum(e[1] for e in self._entries.values())

    def __len__(self) -> int:
        return len(self._entries)

    def acquire(self, prog):
        """The device-resident sampler of ``prog`` (uploaded on a miss), pinned
        until ``release``."""
        d = self._digest(prog)
        with self._lock:
            e = self._entries.get(d)
            if e is not None:
                self._entries.move_to_end(d)
                e[2] += 1
                self.hits += 1
                return d, e[0]
        sampler = B200ProgramSampler(prog, device=self.device)
        nbytes = sum(kc.stats()["image_bytes"] for _, kc in sampler.components)
        with self._lock:
            e = self._entries.get(d)
            if e is not None:  # uploaded concurrently: keep the first
                e[2] += 1
                self.hits += 1
                return d, e[0]
            self.misses += 1
            self._entries[d] = [sampler, nbytes, 1]
            self._evict()
            return d, sampler

    def release(self, digest: str) -> None:
        with self._lock:
            e = self._entries.get(digest)
            if e is not None:
                e[2] -= 1
                self._evict()

    def _evict(self) -> None:
        total = sum(e[1] for e in self._entries.values())
        for d in list(self._entries):
            if total <= self.cache_bytes:
                break
            e = self._entries[d]
            if e[2] > 0:
                continue
            total -= e[1]
            del self._entries[d]
            self.evictions += 1

    def __contains__(self, prog) -> bool:
        return self._digest(prog) in self._entries


class Request:
    """One submitted sample request."""

    def __init__(self, server, rid: int, out: np.ndarray):
        self._srv = server
        self.id = rid
        self.out = out
        self._done = False
        self._error = None
        self.latency_s = None
        self.done_time_s = None

    def done(self) -> bool:
        if self._done:
            return True
        flag = ctypes.c_int32()
        check(self._srv._L.ksim_server_poll(self._srv._h, self.id, ctypes.byref(flag)))
        return bool(flag.value)

    def result(self, timeout: float | None = None) -> np.ndarray:
        """Wait for the request and return its (B, num_outputs) bits."""
        if not self._done:
            L, h = self._srv._L, self._srv._h
            lat, t = ctypes.c_double(), ctypes.c_double()
            ms = -1 if timeout is None else max(0, int(timeout * 1000))
            st = L.ksim_server_wait(h, self.id, ms, ctypes.byref(lat), ctypes.byref(t))
            # the request's own message, before another call replaces it
            msg = (L.ksim_last_error() or b"").decode(errors="replace") if st else ""
            if st == _abi.KSIM_ERR_TIMEOUT:
                flag = ctypes.c_int32()
                if L.ksim_server_poll(h, self.id, ctypes.byref(flag)) == _abi.KSIM_OK:
                    # still queued or running: the wait itself ran out
                    raise TimeoutError(f"request {self.id} not done after {timeout} s")
            self._done = True
            self._srv._retire(self.id)
            if st != _abi.KSIM_OK:
                self._error = _abi.status_error(st, msg)
            else:
                self.latency_s, self.done_time_s = lat.value, t.value
        if self._error is not None:
            raise self._error
        return self.out

    def cancel(self) -> None:
        """Cancel before admission (raises ValueError once on the device)."""
        check(self._srv._L.ksim_server_cancel(self._srv._h, self.id))


class Server:
    """Sample server on one GPU (see the module docstring)."""

    def __init__(self, device: int = 0, arena_bytes: int = 1 << 30, cache_bytes: int = 8 << 30,
                 max_requests: int = 1024, max_jobs: int = 4096, threads: int = 0,
                 slot_bytes: int = 0, ctas_per_sm: int = 0, idle_us: int = 0):
        self._L = lib()
        cfg = _abi.ServerConfig(int(device), int(arena_bytes), int(max_requests), int(max_jobs),
                                int(threads), int(slot_bytes), int(ctas_per_sm), int(idle_us))
        h = ctypes.c_void_p()
        check(self._L.ksim_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self.device = int(device)
        self._cache = ProgramCache(self.device, cache_bytes)
        # buffers and cache pins of requests not yet collected: the native
        # side reads f and writes out until the request is done
        self._inflight: dict = {}
        self._lock = threading.Lock()

    @property
    def cache(self) -> ProgramCache:
        return self._cache

    def submit(self, prog, f_params, seed: int, rng_mode: int = RNG_XORSHIFT,
               out: np.ndarray | None = None) -> Request:
        """Queue ``B200ProgramSampler(prog).sample(f_params, seed)``.  ``f_params``
        may be a row-strided view; ``out`` (optional) receives the bits and
        should be page-locked for the copies to overlap."""
        f = np.asarray(f_params)
        if f.dtype != np.uint8 or f.ndim != 2 or (f.strides[1] != 1 and f.shape[1] > 1):
            f = np.ascontiguousarray(f, dtype=np.uint8)
        if f.ndim != 2:
            raise ValueError("f_params must be 2-D (shots, f parameters)")
        B, n_f = f.shape
        row_stride = int(f.strides[0]) if B > 1 else n_f
        s = _as_u64(seed)
        digest, sampler = self._cache.acquire(prog)
        try:
            n_out = sampler.num_outputs
            if out is None:
                out = np.empty((B, n_out), np.uint8)
            elif out.shape != (B, n_out) or out.dtype != np.uint8 or not out.flags.c_contiguous:
                raise ValueError(f"out must be a C-contiguous uint8 array of shape {(B, n_out)}")
            rid = ctypes.c_int64()
            f_ptr = ctypes.c_void_p(f.ctypes.data) if f.size else None
            check(self._L.ksim_server_submit(self._h, sampler.handle, f_ptr, B, n_f,
                                             max(row_stride, n_f), s, int(rng_mode),
                                             ctypes.c_void_p(out.ctypes.data), ctypes.byref(rid)))
        except BaseException:
            self._cache.release(digest)
            raise
        with self._lock:
            self._inflight[rid.value] = (f, out, sampler, digest)
        return Request(self, rid.value, out)

    def _retire(self, rid: int) -> None:
        with self._lock:
            keep = self._inflight.pop(rid, None)
        if keep is not None:
            self._cache.release(keep[3])

    def sample(self, prog, f_params, seed: int, rng_mode: int = RNG_XORSHIFT) -> np.ndarray:
        return self.submit(prog, f_params, seed, rng_mode).result()

    def stats(self) -> dict:
        st = _abi.ServerStats()
        check(self._L.ksim_server_get_stats(self._h, ctypes.byref(st)))
        d = {name: getattr(st, name) for name, _ in _abi.ServerStats._fields_}
        d.update(cache_programs=len(self._cache), cache_bytes=self._cache.bytes,
                 cache_hits=self._cache.hits, cache_misses=self._cache.misses,
                 cache_evictions=self._cache.evictions)
        return d

    def close(self) -> None:
        """Cancel queued requests, finish running ones and free the server."""
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.ksim_server_destroy(h)
        self._h = None
        with self._lock:
            for keep in self._inflight.values():
                self._cache.release(keep[3])
            self._inflight.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
