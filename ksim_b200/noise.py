"""The per-shot noise draw (the f parameters) on the GPU.

``DeviceChannelSampler(channel_probs, error_transform, seed)`` takes the
arguments of the reference's ``ChannelSampler``
(``src/python/ksim/compile/channels.py:531-576``) and its ``sample(n)``
returns the same kind of (n, num_f) uint8 matrix
(``channels.py:624-658``), drawn by ``ksim_noise_*`` kernels.  At creation
channels over identical error-bit patterns are merged by XOR convolution
(the reference's ``merge_identical_channels``, ``channels.py:398-429``) and
channels of equal firing probability form runs.  The draw is counter-based
(one Philox4x32-10 stream per shot keyed by (seed, shot)): within a run the
next firing channel is found by a geometric skip (one draw, integer
thresholds floor((1 - p)^k 2^32)), a second draw picks the outcome from the
conditional CDF, and the outcome's f pattern is XORed in, so the work per
shot follows the channels that fire.  Per channel the probabilities equal the
reference's to within 2^-32 per threshold, and channels are independent as
in the reference, so the distribution of f is the reference's; the streams
differ (the reference uses numpy's PCG64 with geometric skips along shots).

``B200ProgramSampler.sample_noisy`` draws f on the device and samples from it
in one pipelined call: only the outputs cross PCIe.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import check, lib
from .kokkos_sim import _as_u64

__all__ = ["DeviceChannelSampler", "parity_probability", "channel_patterns"]


def _model_arrays(channel_probs, error_transform):
    probs = [np.ascontiguousarray(np.asarray(p, np.float64)).reshape(-1) for p in channel_probs]
    n_bits = []
    for i, p in enumerate(probs):
        k = int(round(np.log2(len(p)))) if len(p) else -1
        if k < 0 or (1 << k) != len(p):
            raise ValueError(f"channel {i}: {len(p)} probabilities is not a power of two")
        n_bits.append(k)
    T = np.ascontiguousarray(np.asarray(error_transform, np.uint8))
    if T.ndim != 2:
        raise ValueError("error_transform must be 2-D (num_f, num_e)")
    if T.shape[1] != sum(n_bits):
        raise ValueError(f"error_transform has {T.shape[1]} error columns; the channels carry "
                         f"{sum(n_bits)} error bits")
    flat = np.concatenate(probs) if probs else np.zeros(1, np.float64)
    return flat, np.asarray(n_bits or [0], np.int32), len(probs), T


def channel_patterns(channel_probs, error_transform):
    """Per channel: (outcome probabilities, (2^k, num_f) f patterns of the
    outcomes), the outcome's pattern being the XOR of the error_transform
    columns of its error bits."""
    _, n_bits, n_ch, T = _model_arrays(channel_probs, error_transform)
    out, off = [], 0
    for i in range(n_ch):
        k = int(n_bits[i])
        cols = T[:, off:off + k]
        o = np.arange(1 << k)
        bits = ((o[:, None] >> np.arange(k)) & 1).astype(np.int64)
        out.append((np.asarray(channel_probs[i], np.float64), (bits @ cols.T.astype(np.int64)) % 2))
        off += k
    return out


def parity_probability(channel_probs, error_transform, cols) -> float:
    """Exact P(XOR of f[cols] = 1) for independent channels:
    (1 - prod_c (1 - 2 q_c)) / 2 with q_c = P(channel c flips the parity)."""
    cols = np.asarray(cols, np.int64)
    prod = 1.0
    for probs, pats in channel_patterns(channel_probs, error_transform):
        q = float(probs[(pats[:, cols].sum(axis=1) % 2) == 1].sum())
        prod *= 1.0 - 2.0 * q
    return (1.0 - prod) / 2.0


class DeviceChannelSampler:
    """``ChannelSampler`` on the GPU (see the module docstring)."""

    def __init__(self, channel_probs, error_transform, seed: int | None = None, device: int = 0):
        L = lib()
        flat, n_bits, n_ch, T = _model_arrays(channel_probs, error_transform)
        h = ctypes.c_void_p()
        check(L.ksim_noise_create(flat.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                  n_bits.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), n_ch,
                                  _abi.u8ptr(T) if T.size else None, T.shape[0], T.shape[1],
                                  int(device), ctypes.byref(h)))
        self._h, self._L = h, L
        self.num_f = int(T.shape[0])
        self.device = int(device)
        self.seed = _as_u64(int(np.random.default_rng().integers(0, 2**62)) if seed is None
                            else seed)
        self._next_shot = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.ksim_noise_destroy(h)
            self._h = None

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    @property
    def num_channels(self) -> int:
        """Channels that can fire, after merging identical signatures."""
        return int(self._L.ksim_noise_num_channels(self._h))

    def sample(self, num_samples: int = 1) -> np.ndarray:
        """(num_samples, num_f) uint8; successive calls draw successive shots."""
        out = self.sample_at(num_samples, self._next_shot)
        self._next_shot += int(num_samples)
        return out

    def sample_at(self, num_samples: int, shot_offset: int, seed: int | None = None) -> np.ndarray:
        """The rows of shots shot_offset .. shot_offset + num_samples - 1."""
        B = int(num_samples)
        out = np.zeros((B, self.num_f), np.uint8)
        if B and self.num_f:
            check(self._L.ksim_noise_sample(self._h, B, int(shot_offset),
                                            _as_u64(self.seed if seed is None else seed),
                                            _abi.u8ptr(out)))
        return out
