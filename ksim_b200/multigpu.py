"""Multi-GPU sampling: one process per GPU, shots split into contiguous ranges.

Both uniform streams are keyed by the absolute shot index (the xorshift seed
mixing of ``kokkos_sim.cpp:215-217`` and the Philox counter), so rank r
sampling rows [lo, hi) of f with ``shot_offset = lo`` produces exactly rows
[lo, hi) of the one-GPU result.  Nothing crosses NVLink on the data path:
each rank holds its own program replica and its own rows; the only exchange
is the optional gather of result rows to rank 0 at the end (one
``torch.distributed.gather`` of padded uint8 rows, over whatever backend the
process group uses — nccl on GPUs, gloo on the CPU).
"""
from __future__ import annotations

import ctypes

import numpy as np

__all__ = ["shard_range", "ShardedSampler"]


def shard_range(B: int, world: int, rank: int) -> tuple:
    """Rows [lo, hi) of B shots owned by `rank` of `world` (sizes differ by <= 1)."""
    if world < 1 or not 0 <= rank < world or B < 0:
        raise ValueError(f"bad shard request B={B} world={world} rank={rank}")
    base, extra = divmod(B, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def _device_sampler(prog, device):
    """Per-rank sampler on this rank's GPU: (f_rows, seed, rng_mode, shot_offset) -> bits."""
    import torch

    from . import _abi
    from .sampler import B200ProgramSampler
    s = B200ProgramSampler(prog, device=device)
    dev = torch.device("cuda", device)
    L = _abi.lib()

    def run(f_rows, seed, rng_mode, shot_offset):
        B, n_f = f_rows.shape
        out = torch.zeros((B, s.num_outputs), dtype=torch.uint8, device=dev)
        if B == 0 or s.num_outputs == 0:
            return out.cpu().numpy()
        d_f = torch.from_numpy(np.ascontiguousarray(f_rows, np.uint8)).to(dev)
        st = torch.cuda.current_stream(dev)
        _abi.check(L.ksim_program_sample_device(
            s.handle, ctypes.c_void_p(d_f.data_ptr()), B, n_f, int(shot_offset), int(seed),
            int(rng_mode), ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(st.cuda_stream)))
        return out.cpu().numpy()

    return run, s.num_outputs


class ShardedSampler:
    """``sample(f_params, seed)`` split over the ranks of a process group.

    Every rank passes the same full ``f_params`` (or at least its own rows) and
    gets its own rows back from ``sample_local``; ``sample`` also gathers the
    full (B, num_outputs) result on rank 0 (None on the other ranks).
    ``sampler`` overrides the per-rank sampler: a callable
    ``(f_rows, seed, rng_mode, shot_offset) -> bits`` plus ``num_outputs``.
    """

    def __init__(self, prog, group=None, device: int | None = None, sampler=None,
                 num_outputs: int | None = None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        if sampler is None:
            dev = self.rank if device is None else int(device)
            sampler, num_outputs = _device_sampler(prog, dev)
        if num_outputs is None:
            num_outputs = len(prog.output_order)
        self._run = sampler
        self.num_outputs = int(num_outputs)

    def sample_local(self, f_params, seed: int, rng_mode: int = 0) -> tuple:
        """(lo, hi, bits of rows [lo, hi)) for this rank."""
        B = int(f_params.shape[0])
        lo, hi = shard_range(B, self.world, self.rank)
        bits = self._run(f_params[lo:hi], seed, rng_mode, lo)
        return lo, hi, bits

    def sample(self, f_params, seed: int, rng_mode: int = 0, backend_device=None):
        """Full result on rank 0 (None elsewhere).  ``backend_device``: where
        the gathered tensors live (a CUDA device for nccl; None for gloo)."""
        import torch
        B = int(f_params.shape[0])
        lo, hi, bits = self.sample_local(f_params, seed, rng_mode)
        if self.world == 1:
            return bits
        spans = [shard_range(B, self.world, r) for r in range(self.world)]
        rows = max(b - a for a, b in spans)
        pad = np.zeros((rows, self.num_outputs), np.uint8)
        pad[:hi - lo] = bits
        t = torch.from_numpy(pad)
        if backend_device is not None:
            t = t.to(backend_device)
        gather = [torch.empty_like(t) for _ in range(self.world)] if self.rank == 0 else None
        self.dist.gather(t, gather, dst=0, group=self.group)
        if self.rank != 0:
            return None
        return np.concatenate([gather[r].cpu().numpy()[:b - a] for r, (a, b) in enumerate(spans)],
                              axis=0)
