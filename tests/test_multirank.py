"""Shot-split multi-rank sampling, two gloo ranks on the CPU.

Each rank samples its contiguous shot range with shot_offset = its first row
(here through the oracle, the per-rank sampler being injectable) and rank 0
gathers the rows.  The gathered result must equal the one-process result bit
for bit in both uniform streams, for even and uneven splits; a rank that
raises must surface as a failure, not a hang.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from ksim_b200 import synth
from ksim_b200.multigpu import shard_range


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case():
    rng = np.random.default_rng(77)
    prog, n_f = synth.multi_component_program(rng, [(4, 10, 4), (6, 20, 6)])
    f = synth.sample_f(rng, 1001, n_f, 0.05)
    return prog, f


def _worker(rank, world, port, fail_rank):
    import datetime

    import torch.distributed as dist

    from ksim_b200.multigpu import ShardedSampler
    from oracle import oracle as orc
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        prog, f = _case()

        def run(f_rows, seed, mode, off):
            if rank == fail_rank:
                raise RuntimeError(f"rank {rank} failed on purpose")
            return orc.program_sample(prog, f_rows, seed, rng_mode=mode, shot_offset=off)

        ss = ShardedSampler(prog, sampler=run, num_outputs=prog.num_outputs)
        for mode in (0, 1):
            for B in (1001, 2, 0):
                got = ss.sample(f[:B], 4242, mode)
                if rank == 0:
                    want = orc.program_sample(prog, f[:B], 4242, rng_mode=mode)
                    assert got.shape == want.shape and np.array_equal(got, want), (mode, B)
                else:
                    assert got is None
    finally:
        dist.destroy_process_group()


def test_shard_range_partitions():
    for B in (0, 1, 7, 1000, 1001):
        for world in (1, 2, 3, 8):
            spans = [shard_range(B, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == B
            for (a, b), (c, d) in zip(spans, spans[1:]):
                assert b == c and b - a >= d - c >= b - a - 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def test_two_gloo_ranks_match_one_process(oracle_port):
    mp.spawn(_worker, args=(2, _free_port(), -1), nprocs=2, join=True)


def test_failing_rank_is_reported(oracle_port):
    with pytest.raises(Exception):
        mp.spawn(_worker, args=(2, _free_port(), 1), nprocs=2, join=True)
