"""One-call sampling of a compiled circuit: noise -> sample -> (det, obs).

The reference's ``ksim.sample_circuit`` (src/python/ksim/run.py:45-76) does
    compile -> ChannelSampler(channel_probs, error_transform, seed).sample(shots)
    -> KokkosProgramSampler(flat).sample(f, seed) (backend "gpu") or
       sample_flat(flat, f, default_rng(seed)) (backend "cpu")
    -> det = out[:, :num_detectors], obs = out[:, num_detectors:]
and picks the backend in ``_run_sampler`` (run.py:79-91).  Everything after
the compile step is here, on the GPU: the noise draw runs on the device
(``DeviceChannelSampler``, the ChannelSampler model: same channel
probabilities and XOR patterns, a counter-based stream instead of numpy's),
so only the output bits cross PCIe, and the sampler is the B200 drop-in.

The compile step (stim parsing, ZX reduction, stabilizer-rank decomposition:
``ksim.compile``) is not part of this package; ``sample_circuit`` takes it as
a callable, e.g. the reference's ``ksim.compile`` (``__init__.py:75-91``:
circuit -> (FlatProgram, channel_probs, error_transform), through its
compile cache), and ``sample_compiled`` takes its result directly.

Backends: "b200" (alias "gpu", the reference's name for its device path) and
"auto" (b200 when a CUDA device is visible).  There is no CPU sampler in this
package: "cpu" raises ValueError naming the reference's numpy ``sample_flat``,
and "auto" without a device raises instead of falling back.
"""
from __future__ import annotations

import numpy as np

from ._abi import RNG_XORSHIFT, lib

__all__ = ["sample_compiled", "sample_circuit", "resolve_backend"]

_BACKENDS = ("b200", "gpu", "auto", "cpu")


def resolve_backend(backend: str) -> str:
    """The device path for "b200" / "gpu" / "auto"; errors for the rest
    (run.py:79-91 resolves "auto" by trying to import kokkos_sim)."""
    if backend not in _BACKENDS:
        raise ValueError(f"unknown backend {backend!r} (expected b200/gpu/auto)")
    if backend == "cpu":
        raise ValueError("ksim_b200 has no CPU sampler: the CPU path is the reference's numpy "
                         "sample_flat (ksim.sample.sample_flat)")
    if backend == "auto" and lib().ksim_device_count() <= 0:
        raise RuntimeError("backend 'auto': no CUDA device is visible and this package has no CPU path")
    return "b200"


def sample_compiled(flat, channel_probs, error_transform, shots: int, *, seed: int = 42,
                    backend: str = "b200", device: int = 0, rng_mode: int = RNG_XORSHIFT,
                    sampler=None) -> tuple:
    """(det, obs) uint8 arrays of ``shots`` rows for a compiled program.

    ``flat``: the FlatProgram; ``channel_probs`` / ``error_transform``: its
    noise model in ChannelSampler form (an empty ``channel_probs`` means
    noiseless: f is all zero with ``error_transform.shape[0]`` columns, as in
    run.py:67-72).  ``seed`` seeds both the noise draw and the sampler, as in
    the reference.  ``sampler`` (optional): a ``B200ProgramSampler`` of
    ``flat`` to reuse across calls instead of uploading the program again."""
    from .noise import DeviceChannelSampler
    from .sampler import B200ProgramSampler
    resolve_backend(backend)
    shots = int(shots)
    if shots < 0:
        raise ValueError("shots must be >= 0")
    s = sampler if sampler is not None else B200ProgramSampler(flat, device=device)
    T = np.asarray(error_transform, np.uint8)
    if len(channel_probs):
        noise = DeviceChannelSampler(channel_probs, T, seed=seed, device=device)
        out = s.sample_noisy(noise, shots, seed, noise_seed=seed, rng_mode=rng_mode)
    else:
        n_f = T.shape[0] if T.size else 0
        out = s.sample(np.zeros((shots, n_f), np.uint8), seed, rng_mode=rng_mode)
    nd = int(flat.num_detectors)
    return out[:, :nd].astype(np.uint8), out[:, nd:].astype(np.uint8)


def sample_circuit(circuit, shots: int, *, compile_fn, seed: int = 42, backend: str = "b200",
                   device: int = 0, rng_mode: int = RNG_XORSHIFT) -> tuple:
    """``ksim.sample_circuit`` with a pluggable compile step:
    ``compile_fn(circuit) -> (flat, channel_probs, error_transform)``."""
    resolve_backend(backend)
    flat, channel_probs, error_transform = compile_fn(circuit)
    return sample_compiled(flat, channel_probs, error_transform, shots, seed=seed, backend=backend,
                           device=device, rng_mode=rng_mode)
