"""Batched form: many programs in one persistent, graph-captured launch.

Each program's result must be bit-identical to the oracle's (and so to the
one-program-per-launch path) for the same seed, whatever shares the launch,
under every launch shape the autotuner may pick, with and without the graph.
"""
from __future__ import annotations

import numpy as np
import pytest

from ksim_b200 import synth

pytestmark = pytest.mark.gpu


def _mixed_programs(seed=40):
    rng = np.random.default_rng(seed)
    progs, shots, fs = [], [], []
    specs = [
        [(5, 0, 4)], [(12, 30, 6)], [(40, 64, 10)], [(8, 130, 5)],       # W = 1, 1, 2, 3
        [(3, 5, 3), (6, 12, 6), (2, 0, 2)],                             # multi-component
        [(20, 300, 4)],                                                 # W = 5 (second class)
        [(1, 0, 1)], [(30, 60, 12)], [(10, 20, 8)], [(4, 4, 2)],
    ]
    for sp in specs:
        if len(sp) == 1:
            n_out, F, t = sp[0]
            comp = synth.random_component(rng, n_out=n_out, F=F, t=t, f_prob=0.05)
            prog, nf = synth.single_component_program(comp), F
        else:
            prog, nf = synth.multi_component_program(rng, sp)
        b = int(rng.integers(1, 3000))
        progs.append(prog)
        shots.append(b)
        fs.append(synth.sample_f(rng, b, nf, 0.05))
    shots[6] = 0  # an empty job
    fs[6] = fs[6][:0]
    return progs, shots, fs


@pytest.fixture(scope="module")
def mixed():
    return _mixed_programs()


def _classes(progs, shots):
    """(W class, term-path class) of every component with work: W above 4 is
    one class, below it each W with 32-bit / hybrid / general terms."""
    from ksim_b200 import perfmodel
    from ksim_b200.kokkos_sim import Component
    out = set()
    for prog, b in zip(progs, shots):
        for comp in prog.components:
            if b == 0 or len(comp.graphs) <= 1:
                continue
            w = Component(comp.graphs, int(np.asarray(comp.f_selection).shape[0])).words
            r = perfmodel.component_work(comp)
            terms = r["narrow_terms"] + r["wide_terms"] + r["exact_terms"] + r["hybrid_terms"]
            paths = (0 if r["narrow_terms"] == terms else
                     1 if r["narrow_terms"] + r["hybrid_terms"] == terms else 2)
            out.add((w, paths) if w <= 4 else ("wide",))
    return out


def _oracle(oracle_port, progs, fs, seeds, mode):
    return [oracle_port.program_sample(p, f, s, rng_mode=mode) for p, f, s in zip(progs, fs, seeds)]


@pytest.mark.parametrize("mode", [0, 1])
def test_batch_matches_oracle(cuda_device, oracle_port, mixed, mode):
    from ksim_b200.batch import BatchSampler
    progs, shots, fs = mixed
    seeds = [17 + 1000 * i for i in range(len(progs))]
    bs = BatchSampler(progs, shots, seeds=seeds, rng_mode=mode, n_f=[f.shape[1] for f in fs])
    # one persistent kernel per (W, term paths) class with work
    assert bs.info()["launches"] == len(_classes(progs, shots))
    got = bs.sample(fs)
    want = _oracle(oracle_port, progs, fs, seeds, mode)
    for i, (g, w) in enumerate(zip(got, want)):
        assert np.array_equal(g, w), i


def test_batch_shapes_graph_and_reseed(cuda_device, oracle_port, mixed):
    from ksim_b200.batch import BatchSampler
    progs, shots, fs = mixed
    seeds = list(range(3, 3 + len(progs)))
    want = _oracle(oracle_port, progs, fs, seeds, 0)
    bs = BatchSampler(progs, shots, seeds=seeds, n_f=[f.shape[1] for f in fs])
    bs.set_inputs(fs)
    for tuning in ({"threads": 64, "slot_bytes": 8192, "ctas_per_sm": 1},
                   {"threads": 128, "slot_bytes": 32768, "ctas_per_sm": 0},
                   {"threads": 256, "slot_bytes": 16384, "ctas_per_sm": 2}):
        bs._build(tuning)
        for _ in range(2):  # graph replay twice
            bs.launch()
            for i, (g, w) in enumerate(zip(bs.results(), want)):
                assert np.array_equal(g, w), (tuning, i)
    # reseed between replays of the same graph
    seeds2 = [s * 7 + 1 for s in seeds]
    bs.set_seeds(seeds2)
    bs.launch()
    for g, w in zip(bs.results(), _oracle(oracle_port, progs, fs, seeds2, 0)):
        assert np.array_equal(g, w)
    # no graph
    nog = BatchSampler(progs, shots, seeds=seeds, use_graph=False, n_f=[f.shape[1] for f in fs])
    for g, w in zip(nog.sample(fs), want):
        assert np.array_equal(g, w)


def test_batch_equals_plain_launches(cuda_device, mixed):
    from ksim_b200.batch import BatchSampler
    progs, shots, fs = mixed
    bs = BatchSampler(progs, shots, seeds=[5] * len(progs), n_f=[f.shape[1] for f in fs])
    batched = bs.sample(fs)
    bs.launch_plain()
    plain = bs.results()
    for a, b in zip(batched, plain):
        assert np.array_equal(a, b)


def test_autotuner_picks_a_valid_shape(cuda_device, tmp_path, monkeypatch, mixed):
    from ksim_b200.batch import BatchSampler, tune_cache_path
    monkeypatch.setenv("KSIM_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    progs, shots, fs = mixed
    bs = BatchSampler(progs, shots, n_f=[f.shape[1] for f in fs])
    rec = bs.tune(candidates=[{"threads": 128, "slot_bytes": 16384, "ctas_per_sm": 0},
                              {"threads": 256, "slot_bytes": 16384, "ctas_per_sm": 0}])
    assert rec["tuning"]["threads"] in (128, 256) and rec["ms"] > 0
    assert tune_cache_path().exists()
    again = BatchSampler(progs, shots, n_f=[f.shape[1] for f in fs]).tune()
    assert again["tuning"] == rec["tuning"]
