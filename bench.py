#!/usr/bin/env python
"""Benchmark of the B200 sampling hot path (FlatProgram -> samples).

``python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]``

One step = sampling every shot of the workload once (one pass of the hot
path over one batch).  Default workload: the medium plain-method program (40
outputs, t = 12 T gates, F = 64 noise parameters, 1e6 shots per GPU; seeded
synthetic FlatProgram of that shape, ksim_b200.synth.config(2)).  Prints one
JSON line on rank 0.

* ``value``: shots/s of the whole job, inputs resident in HBM, kernel time by
  CUDA events on the launching stream, L2 flushed (256 MiB write) between
  steps, max over ranks.
* ``e2e``: the same metric through the public drop-in API
  (``B200ProgramSampler.sample``) from pinned host memory, host<->device
  copies inside the timed region.
* ``roofline``: integer-ALU bound; algorithmic int32 ops per launch
  (ksim_b200.perfmodel) / event time vs the integer-pipe peak measured on
  this GPU by ksim_measure_int_peak.
* ``cpu_baseline``: the reference's own zx_eval.hpp (oracle/_ref) or its C
  restatement, all host threads, on a bounded shot sample.

``--impl reference`` times that CPU implementation alone on the same workload
(rank 0 only under torchrun).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = ("shots/sec at 1 B200, batched+served vs plain, bit-exact Z[ω]; p50/p99 latency")
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", type=int, default=2, choices=(1, 2, 4))
    ap.add_argument("--shots", type=int, default=0, help="override shots per GPU")
    ap.add_argument("--rng", type=int, default=0, help="0 xorshift (kokkos_sim), 1 philox")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def workload(args):
    from ksim_b200 import synth
    w = synth.config(args.workload)
    shots = args.shots or w.shots
    rng = np.random.default_rng(w.seed + 1)
    f = synth.sample_f(rng, shots, w.n_f, w.f_prob)
    return w, shots, f


def cpu_reference_rate(prog, f, seed, rng_mode, target_s, max_shots):
    """Shots/s of the CPU reference implementation on a bounded prefix."""
    from oracle import oracle as orc
    if not orc.PORT_LIB.exists():
        orc.build()
    kind = "reference" if orc.RefOracle.available() else "port"
    cls = orc.RefOracle if kind == "reference" else orc.PortOracle
    threads = os.cpu_count() or 1
    n = min(256, max_shots)
    t0 = time.perf_counter()
    orc.program_sample(prog, f[:n], seed, rng_mode, oracle_cls=cls, n_threads=threads)
    dt = time.perf_counter() - t0
    n2 = int(min(max_shots, max(n, n * target_s / max(dt, 1e-6))))
    t0 = time.perf_counter()
    orc.program_sample(prog, f[:n2], seed, rng_mode, oracle_cls=cls, n_threads=threads)
    dt = time.perf_counter() - t0
    return n2 / dt, kind, threads, n2, dt


def run_reference(args):
    world, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return
    w, shots, f = workload(args)
    from oracle import oracle as orc
    if not orc.PORT_LIB.exists():
        orc.build()
    kind = "reference" if orc.RefOracle.available() else "port"
    cls = orc.RefOracle if kind == "reference" else orc.PortOracle
    threads = os.cpu_count() or 1
    # size each step to ~3 s of CPU work so warmup + steps stay within minutes
    n = min(256, shots)
    t0 = time.perf_counter()
    orc.program_sample(w.program, f[:n], 1234, args.rng, oracle_cls=cls, n_threads=threads)
    per = (time.perf_counter() - t0) / n
    step_shots = int(max(64, min(shots, 3.0 / max(per, 1e-9))))
    for i in range(args.warmup):
        orc.program_sample(w.program, f[:step_shots], 1234 + i, args.rng, oracle_cls=cls,
                           n_threads=threads)
    times = []
    for i in range(args.steps):
        t0 = time.perf_counter()
        orc.program_sample(w.program, f[:step_shots], 99 + i, args.rng, oracle_cls=cls,
                           n_threads=threads)
        times.append(time.perf_counter() - t0)
    value = step_shots * len(times) / sum(times)
    sample = (f"first {step_shots} of {shots} shots of {w.name} per step "
              f"({'zx_eval.hpp compiled unmodified + restated kokkos_sim loop' if kind == 'reference' else 'C restatement of zx_eval.hpp'}, OpenMP)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "shots/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": {"workload": w.name, "shots_per_gpu": shots, "step_shots": step_shots},
            "cpu_baseline": {"value": value, "unit": "shots/s", "cores": threads, "kind": kind,
                             "sample": sample},
            "e2e": {"value": value, "unit": "shots/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    world, rank, local = dist_setup(args)
    import torch
    torch.cuda.set_device(local)
    from ksim_b200 import _abi, perfmodel
    from ksim_b200.sampler import B200ProgramSampler
    L = _abi.lib()

    w, shots, f = workload(args)
    prog = w.program
    sampler = B200ProgramSampler(prog, device=local)
    n_out = sampler.num_outputs
    n_f = f.shape[1]
    work = perfmodel.program_work(prog)

    dev = torch.device("cuda", local)
    d_f = torch.from_numpy(f).to(dev)
    d_out = torch.zeros((shots, n_out), dtype=torch.uint8, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    offset = rank * shots  # weak scaling: each GPU samples its own shot range

    def launch(seed):
        _abi.check(L.ksim_program_sample_device(
            sampler.handle, ctypes.c_void_p(d_f.data_ptr()), shots, n_f, offset, seed, args.rng,
            ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(stream.cuda_stream)))

    peak = ctypes.c_double()
    _abi.check(L.ksim_measure_int_peak(local, ctypes.byref(peak), None))

    for i in range(args.warmup):
        launch(1000 + i)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            flush.zero_()
            evs[i][0].record(stream)
            launch(2000 + i)
            evs[i][1].record(stream)
        torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = max_over_ranks(sum(step_ms), world)
    value = world * shots * args.steps / (total_ms / 1e3)
    ms_per_step = total_ms / args.steps

    # end to end through the drop-in API from pinned host memory
    f_pin = torch.from_numpy(f).pin_memory().numpy()
    for i in range(max(1, args.warmup)):
        sampler.sample(f_pin, 3000 + i, rng_mode=args.rng)
    barrier(world)
    e2e_t = []
    for i in range(args.steps):
        t0 = time.perf_counter()
        out = sampler.sample(f_pin, 4000 + i, rng_mode=args.rng)
        e2e_t.append(time.perf_counter() - t0)
    e2e_total = max_over_ranks(sum(e2e_t), world)
    e2e_value = world * shots * args.steps / e2e_total

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, kind, cores, n, dt = cpu_reference_rate(prog, f, 2000, args.rng, args.cpu_seconds,
                                                      shots)
        cpu = {"value": rate, "unit": "shots/s", "cores": cores, "kind": kind,
               "sample": f"first {n} shots of {w.name}, {dt:.1f} s on {cores} threads"}

    if rank == 0:
        mean_s = (sum(step_ms) / len(step_ms)) / 1e3
        achieved = work["ops"] * shots / mean_s
        hbm_bytes = shots * (work["in_bytes"] + work["out_bytes"])
        line = {
            "metric": METRIC, "value": value, "unit": "shots/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic",
            "config": {"workload": f"{w.name}: {n_out} outputs, F={n_f}, "
                                   f"{work['terms']} terms/shot over {work['graphs']} graphs",
                       "shots_per_gpu": shots,
                       "rng": "xorshift (kokkos_sim stream)" if args.rng == 0 else "philox4x32-10",
                       "l2": "flushed between steps (256 MiB write)",
                       "parallelism": f"shot-split x{world}"},
            "e2e": {"value": e2e_value, "unit": "shots/s", "h2d_bytes_per_step": int(f.nbytes),
                    "d2h_bytes_per_step": int(shots * n_out)},
            "roofline": {"bound": "alu", "achieved": achieved / 1e9, "peak": peak.value / 1e9,
                         "unit": "Gop/s (int32)", "frac": achieved / peak.value,
                         "traffic": None,
                         "ops_per_shot": work["ops"], "hbm_gbs": hbm_bytes / mean_s / 1e9,
                         "peak_source": "ksim_measure_int_peak on this GPU (burst)"},
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "gpu_launches": args.steps * len(prog.components),
            "step_ms": step_ms,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
