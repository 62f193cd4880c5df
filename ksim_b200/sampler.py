"""``B200ProgramSampler`` — drop-in for the reference's ``KokkosProgramSampler``.

``B200ProgramSampler(prog).sample(f_params, seed)`` has the signature and the
result of ``KokkosProgramSampler`` (``src/python/ksim/sample/sampler.py:46-67``)
and of the numpy ``sample_flat`` (``sample/evaluate.py:69-87``): one native
component per ``FlatComponent``, component ``k`` seeded with
``seed + 0x9E37*k``, outputs concatenated and permuted by
``argsort(output_order)``.  Here the f_selection gather, every component's
kernel and the permutation run on the device in one native call.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import RNG_PHILOX, RNG_XORSHIFT, check, lib
from .kokkos_sim import Component, _as_u64
from .program import graph_to_dict

__all__ = ["B200ProgramSampler", "KokkosProgramSampler", "graph_to_dict"]


class B200ProgramSampler:
    """GPU sampler for a FlatProgram (any object with the FlatProgram fields)."""

    def __init__(self, prog, device: int = -1):
        L = lib()
        self.prog = prog
        self.components = []
        sels = []
        for comp in prog.components:
            sel = np.ascontiguousarray(np.asarray(comp.f_selection), dtype=np.int32).reshape(-1)
            kc = Component([graph_to_dict(g) for g in comp.graphs], int(sel.shape[0]),
                           device=device)
            self.components.append((comp, kc))
            sels.append(sel)
        self._sels = sels
        order = np.ascontiguousarray(np.asarray(prog.output_order), dtype=np.int32).reshape(-1)
        self._order = order
        n = len(self.components)
        handles = (ctypes.c_void_p * max(n, 1))(*[kc.handle.value for _, kc in self.components])
        sel_ptrs = (ctypes.POINTER(ctypes.c_int32) * max(n, 1))(*[_abi.i32ptr(s) for s in sels])
        sel_len = np.array([s.shape[0] for s in sels] or [0], np.int32)
        h = ctypes.c_void_p()
        check(L.ksim_program_create(handles, n, sel_ptrs, _abi.i32ptr(sel_len), _abi.i32ptr(order),
                                    int(order.shape[0]), ctypes.byref(h)))
        self._h = h
        self._L = L
        self.num_outputs = int(order.shape[0])
        self.min_f_cols = int(L.ksim_program_min_f_cols(h))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.ksim_program_destroy(h)
            self._h = None

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def sample(self, f_params: np.ndarray, seed: int, rng_mode: int = RNG_XORSHIFT,
               out: np.ndarray | None = None) -> np.ndarray:
        """KokkosProgramSampler.sample.  ``out`` (optional): a C-contiguous
        (B, num_outputs) uint8 array to fill, e.g. page-locked memory so the
        device-to-host copies run asynchronously."""
        f = np.ascontiguousarray(f_params, dtype=np.uint8)
        if f.ndim != 2:
            raise ValueError("f_params must be 2-D (shots, f parameters)")
        B = f.shape[0]
        s = _as_u64(seed)
        _as_u64(s + 0x9E37 * max(len(self.components) - 1, 0))  # per-component seeds stay uint64
        if f.shape[1] < self.min_f_cols:
            raise IndexError(f"f_params has {f.shape[1]} columns; f_selection needs "
                             f"{self.min_f_cols}")
        if out is None:
            out = np.zeros((B, self.num_outputs), np.uint8)
        elif out.shape != (B, self.num_outputs) or out.dtype != np.uint8 or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous uint8 array of shape {(B, self.num_outputs)}")
        if B == 0 or self.num_outputs == 0:
            return out
        check(self._L.ksim_program_sample(self._h, _abi.u8ptr(f), B, f.shape[1], s, int(rng_mode),
                                          _abi.u8ptr(out)))
        return out


    def sample_packed(self, f_packed: np.ndarray, n_f_cols: int, seed: int,
                      rng_mode: int = RNG_XORSHIFT, out: np.ndarray | None = None) -> np.ndarray:
        """``sample`` with bit-packed rows: ``f_packed`` is (B, ceil(n_f_cols/8))
        uint8 as ``np.packbits(f, axis=1, bitorder="little")``; returns
        (B, ceil(num_outputs/8)) packed the same way.  ``out`` (optional): a
        C-contiguous array of that shape to fill, e.g. page-locked memory."""
        f = np.ascontiguousarray(f_packed, dtype=np.uint8)
        if f.ndim != 2 or f.shape[1] != (int(n_f_cols) + 7) // 8:
            raise ValueError(f"f_packed must have {(int(n_f_cols) + 7) // 8} bytes per row")
        if n_f_cols < self.min_f_cols:
            raise IndexError(f"f_params has {n_f_cols} columns; f_selection needs {self.min_f_cols}")
        B = f.shape[0]
        shape = (B, (self.num_outputs + 7) // 8)
        if out is None:
            out = np.zeros(shape, np.uint8)
        elif out.shape != shape or out.dtype != np.uint8 or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous uint8 array of shape {shape}")
        if B == 0 or self.num_outputs == 0:
            return out
        check(self._L.ksim_program_sample_packed(self._h, _abi.u8ptr(f), B, int(n_f_cols), _as_u64(seed),
                                                 int(rng_mode), _abi.u8ptr(out)))
        return out


    def sample_noisy(self, noise, shots: int, seed: int, noise_seed: int | None = None,
                     rng_mode: int = RNG_XORSHIFT, out: np.ndarray | None = None) -> np.ndarray:
        """Draw f with ``noise`` (a ``DeviceChannelSampler``, shots 0..shots-1 of
        its stream ``noise_seed``, default its own seed) and sample from it, all
        on the device; equals ``sample(noise.sample_at(shots, 0), seed)``."""
        B = int(shots)
        ns = _as_u64(noise.seed if noise_seed is None else noise_seed)
        if out is None:
            out = np.zeros((B, self.num_outputs), np.uint8)
        elif out.shape != (B, self.num_outputs) or out.dtype != np.uint8 or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous uint8 array of shape {(B, self.num_outputs)}")
        if B == 0 or self.num_outputs == 0:
            return out
        check(self._L.ksim_program_sample_noisy(self._h, noise.handle, B, ns, _as_u64(seed),
                                                int(rng_mode), _abi.u8ptr(out)))
        return out


KokkosProgramSampler = B200ProgramSampler
