"""GPU parity on the benchmark configurations themselves.

The synthetic stand-ins of the five workloads (``ksim_b200.synth``) run
through the drop-in API, the batched launch and the server, and every sampled
bit and |A_k| must equal the reference's own ``zx_eval.hpp`` (``oracle/_ref``,
compiled unmodified, driven by the restated kokkos_sim loop,
kokkos_sim.cpp:214-230), in both uniform streams:

* cfg1 (5 outputs, t = 4, noiseless): all 1e5 shots;
* cfg2 (40 outputs, t = 12, F = 64) and cfg4 (16 parity outputs, t = 20,
  F = 56): a 32 Ki-shot prefix through ``B200ProgramSampler.sample`` and a
  4 Ki-shot slice at shot index 900,000 through the device entry point;
* cfg3: the whole 64-program batch in one persistent launch, the 8 programs
  with the most terms checked on a prefix and on their last rows;
* cfg5: requests for 10 programs of the serving pool submitted together, so
  their tiles interleave in the device-resident loop;
* one plain program with a 4-word (193-256 bit) parameter vector.

Tolerance: none (bit-exact bits and |A_k| doubles).
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from helpers import same_bits
from ksim_b200 import synth

pytestmark = pytest.mark.gpu


def _device_sample(kc, f, seed, mode, shot_offset=0):
    """ksim_component_sample_device with torch buffers -> (bits, |A_k|)."""
    import torch
    from ksim_b200 import _abi
    B = f.shape[0]
    d_f = torch.from_numpy(np.ascontiguousarray(f, np.uint8)).cuda()
    d_out = torch.zeros((B, max(kc.n_out, 1)), dtype=torch.uint8, device="cuda")
    d_amp = torch.zeros((B, kc.n_out + 1), dtype=torch.float64, device="cuda")
    _abi.check(_abi.lib().ksim_component_sample_device(
        kc.handle, ctypes.c_void_p(d_f.data_ptr()), B, shot_offset, seed, mode,
        ctypes.c_void_p(d_out.data_ptr()), max(kc.n_out, 1), 0, ctypes.c_void_p(d_amp.data_ptr()),
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    return d_out.cpu().numpy()[:, :kc.n_out], d_amp.cpu().numpy()


def _check_single(w, ref, f, shot_offset, seeds=(2024, 2**63 + 99)):
    """Drop-in call (offset 0) or device call (any offset) of a one-component
    workload against the reference oracle: bits and |A_k|."""
    from ksim_b200.sampler import B200ProgramSampler
    prog = w.program
    comp = prog.components[0]
    F = int(np.asarray(comp.f_selection).shape[0])
    sampler = B200ProgramSampler(prog, device=0)
    kc = sampler.components[0][1]
    oc = ref(comp.graphs, F)
    f_sel = np.ascontiguousarray(f[:, np.asarray(comp.f_selection, np.int64)])
    for seed in seeds:
        for mode in (0, 1):
            want, want_amp = oc.sample(f_sel, seed, mode, shot_offset=shot_offset, return_amp=True)
            if shot_offset == 0:
                got = sampler.sample(f, seed, rng_mode=mode)
                assert np.array_equal(got, want[:, np.argsort(prog.output_order)]), (seed, mode)
            bits, amp = _device_sample(kc, f_sel, seed, mode, shot_offset)
            assert np.array_equal(bits, want[:, :kc.n_out]), (seed, mode, shot_offset)
            assert same_bits(amp, want_amp), (seed, mode, shot_offset)


def test_cfg1_all_shots(cuda_device, ref_oracle):
    w = synth.config(1)
    f = np.zeros((w.shots, 0), np.uint8)
    _check_single(w, ref_oracle, f, 0)


@pytest.mark.parametrize("cfg", [2, 4])
def test_cfg2_cfg4_prefix_and_far_slice(cuda_device, ref_oracle, cfg):
    w = synth.config(cfg)
    assert w.program.components[0] is not None
    rng = np.random.default_rng(w.seed + 1)
    f = synth.sample_f(rng, 32768, w.n_f, w.f_prob)
    _check_single(w, ref_oracle, f, 0, seeds=(2024,))
    far = synth.sample_f(rng, 4096, w.n_f, w.f_prob)
    _check_single(w, ref_oracle, far, 900_000, seeds=(2**63 + 99,))


def test_cfg3_batch_largest_programs(cuda_device, oracle_module, ref_oracle):
    from ksim_b200.batch import BatchSampler
    ws = synth.batched_workloads()
    rng = np.random.default_rng(3001)
    fs = [synth.sample_f(rng, w.shots, w.n_f, w.f_prob) for w in ws]
    terms = [sum(int(g.pf_phase_idx.shape[0]) for g in w.program.components[0].graphs) for w in ws]
    largest = np.argsort(terms)[::-1][:8]
    for mode in (0, 1):
        bs = BatchSampler([w.program for w in ws], [w.shots for w in ws],
                          seeds=[w.seed for w in ws], rng_mode=mode, device=0,
                          n_f=[w.n_f for w in ws])
        outs = bs.sample(fs)
        for i in largest:
            w, f, got = ws[i], fs[i], outs[i]
            head = min(2048, w.shots)
            want = oracle_module.program_sample(w.program, f[:head], w.seed, mode, oracle_cls=ref_oracle)
            assert np.array_equal(got[:head], want), (w.name, mode)
            tail = min(512, w.shots - head)
            if tail > 0:
                lo = w.shots - tail
                want = oracle_module.program_sample(w.program, f[lo:], w.seed, mode,
                                                    oracle_cls=ref_oracle, shot_offset=lo)
                assert np.array_equal(got[lo:], want), (w.name, mode, "tail")


def test_cfg5_pool_requests_in_the_mix(cuda_device, oracle_module, ref_oracle):
    from ksim_b200.serve import Server
    pool = synth.serving_pool()
    rng = np.random.default_rng(5556)
    picks = list(range(0, 200, 20))
    reqs = []
    for pi in picks:
        for _ in range(2):
            B = int(round(np.exp(rng.uniform(np.log(1e2), np.log(6e3)))))
            w = pool[pi]
            reqs.append((pi, synth.sample_f(rng, B, w.n_f, w.f_prob), int(rng.integers(0, 2**62)),
                         int(rng.integers(0, 2))))
    with Server(device=0, idle_us=2000) as srv:
        hs = [srv.submit(pool[pi].program, f, seed, mode) for pi, f, seed, mode in reqs]
        got = [h.result(timeout=300) for h in hs]
        st = srv.stats()
    assert st["failed"] == 0 and st["completed"] == len(reqs)
    for (pi, f, seed, mode), g in zip(reqs, got):
        want = oracle_module.program_sample(pool[pi].program, f, seed, mode, oracle_cls=ref_oracle)
        assert np.array_equal(g, want), (pi, seed, mode)


def test_plain_sampler_four_word_vectors(cuda_device, ref_oracle):
    from ksim_b200.kokkos_sim import Component
    rng = np.random.default_rng(4444)
    comp = synth.random_component(rng, n_out=12, F=200, t=9, f_prob=0.03)
    kc = Component(comp.graphs, 200)
    assert kc.words == 4
    oc = ref_oracle(comp.graphs, 200)
    f = synth.sample_f(rng, 6000, 200, 0.03)
    for mode in (0, 1):
        want, want_amp = oc.sample(f, 31, mode, return_amp=True)
        assert np.array_equal(kc.sample(f, 31, rng_mode=mode), want)
        bits, amp = _device_sample(kc, f, 31, mode, 123_456)
        want, want_amp = oc.sample(f, 31, mode, shot_offset=123_456, return_amp=True)
        assert np.array_equal(bits, want[:, :kc.n_out]) and same_bits(amp, want_amp)
