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
* ``roofline``: instruction-issue bound: thread instructions per shot (one
  ncu capture, NCU_THREAD_INST_PER_SHOT) x shots/s over SMs x 4 issue slots
  x 32 lanes x the sampled SM clock; beside it both int32 op models (the
  formulation's and the reference algorithm's) against two measured integer
  peaks (the sampler's add/shift/logic mix and add/logic alone).
* ``parity``: the first rows of the last timed output and of the last e2e
  output against the reference's own zx_eval.hpp (oracle/_ref).
* ``cpu_baseline``: the reference's own zx_eval.hpp (oracle/_ref) or its C
  restatement, all host threads, on a bounded shot sample;
  ``cpu_baseline_numpy``: the reference's numpy sample_flat (restated in
  oracle/numpy_flat.py), one process, on a bounded prefix.
* ``legs``: cfg1 (5 outputs, t = 4, 1e5 shots) and cfg4 (16 parity outputs,
  t = 20, 1e6 shots) through the same plain path, with e2e and parity.
* ``batched`` (1 GPU): 64 seeded programs (qubits U[8,60], t U[2,16], shots
  log-uniform 1e3-1e5) in one persistent graph-replayed launch, autotuned,
  vs 64 plain one-program launches; device time, L2 flushed, bit identity
  of the two checked.
* ``served`` (1 GPU): 10 000 Poisson requests over a 200-program pool at
  80 % of the batched capacity of the same request mix (its first requests
  run as one autotuned batch) through the continuous-batching server:
  shots/s and p50/p99 latency (arrival -> bits in host memory, host clock),
  vs the same stream through plain per-request calls.

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
# DRAM bytes per shot of the plain kernel, from one ncu capture of
# k_sample on the same workload at 262,144 shots (dram__bytes_read.sum +
# dram__bytes_write.sum), plus the output row the capture's L2 absorbed;
# scaled to a launch by its shots (the capture's command and figures are kept
# with the ncu summaries under profiles/).
NCU_DRAM_BYTES_PER_SHOT = {"cfg2-medium-40q-t12": 67.4 + 40.0, "cfg4-large-rank-85q-t20": 61.1 + 16.0}
# Thread instructions per shot of the plain kernel on the same workload, from
# one ncu capture (smsp__thread_inst_executed.sum / shots of the captured
# launch); the issue roofline of the bench line is this times shots/s over
# the SMs' issue ceiling (capture command and figures: the ncu summaries
# under profiles/).
NCU_THREAD_INST_PER_SHOT = {"cfg2-medium-40q-t12": 138386, "cfg4-large-rank-85q-t20": 201817}
# Thread instructions of one cfg3 batch (its five class kernels, one ncu
# capture at the default launch shape: 128 threads, 14 KiB slots); the
# batched leg's issue fraction is this over its timed batch and the issue
# ceiling (capture command and figures: the ncu summaries under profiles/).
NCU_THREAD_INST_PER_BATCH = 88.83e9
NCU_BATCH_SHAPE = {"threads": 128, "slot_bytes": 14336, "ctas_per_sm": 0}
# Gate locations of the workloads' circuits (qubits x depth): one
# single-qubit Pauli channel each in the noisy end-to-end leg.
NOISE_LOCATIONS = {"cfg2-medium-40q-t12": 40 * 200, "cfg4-large-rank-85q-t20": 85 * 600}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", type=int, default=2, choices=(1, 2, 4))
    ap.add_argument("--shots", type=int, default=0, help="override shots per GPU")
    ap.add_argument("--rng", type=int, default=0, help="0 xorshift (kokkos_sim), 1 philox")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched (64-program) leg")
    ap.add_argument("--no-served", action="store_true", help="skip the served (request stream) leg")
    ap.add_argument("--requests", type=int, default=10_000, help="requests of the served leg")
    ap.add_argument("--load", type=float, default=0.8,
                    help="served arrival rate as a fraction of the batched capacity measured "
                         "on the request mix")
    ap.add_argument("--legs", default="1,4",
                    help="extra plain workloads timed beside the headline one (config numbers)")
    ap.add_argument("--parity-shots", type=int, default=4096,
                    help="shots of each timed output checked against the reference oracle")
    ap.add_argument("--numpy-seconds", type=float, default=8.0,
                    help="CPU seconds of the numpy sample_flat baseline")
    ap.add_argument("--serve-threads", type=int, default=0,
                    help="threads per CTA of the serving loop (0: the library default)")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons every 10 ms; summary() keeps the
    samples taken inside the timed region (between begin() and end())."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int, period_ms: int = 10):
        self.index = index
        self.period_ms = period_ms
        self.proc = None
        self.lines = []  # (perf_counter, line)
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", str(self.period_ms)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            deadline = time.perf_counter() + 3.0   # the first sample takes a moment
            while not self.lines and time.perf_counter() < deadline:
                time.sleep(0.01)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def begin(self):
        self.t0 = time.perf_counter()

    def end(self):
        self.t1 = time.perf_counter()

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
        t0 = self.t0 if self.t0 is not None else float("-inf")
        t1 = self.t1 if self.t1 is not None else float("inf")
        for ts, ln in self.lines:
            if not t0 <= ts <= t1 + self.period_ms / 1e3:
                continue
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
                "reasons": sorted(reasons), "samples": len(sm),
                "period_ms": self.period_ms}


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


def cpu_model() -> str:
    """The host CPU's model name (for the CPU-baseline records)."""
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.lower().startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def parity_check(prog, f_rows, bits, seed, rng_mode, shot_offset=0):
    """Compare sampled rows with the reference's own zx_eval.hpp (oracle/_ref,
    or its C restatement where that is not built), all host threads."""
    from oracle import oracle as orc
    if not orc.PORT_LIB.exists():
        orc.build()
    cls = orc.RefOracle if orc.RefOracle.available() else orc.PortOracle
    want = orc.program_sample(prog, f_rows, seed, rng_mode, oracle_cls=cls, shot_offset=shot_offset)
    return {"shots": int(f_rows.shape[0]), "ok": bool(np.array_equal(bits, want)),
            "checker": "oracle/_ref (zx_eval.hpp)" if cls is orc.RefOracle else "C restatement"}


def numpy_baseline(prog, f, target_s):
    """Shots/s of the reference's numpy sample_flat (restated in
    oracle/numpy_flat.py, one process) on a prefix sized to ~target_s."""
    from oracle import numpy_flat as nf
    import warnings
    n = min(32, f.shape[0])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        t0 = time.perf_counter()
        nf.sample_flat(prog, f[:n], np.random.default_rng(1))
        dt = time.perf_counter() - t0
        n2 = int(min(f.shape[0], max(n, n * target_s / max(dt, 1e-6))))
        t0 = time.perf_counter()
        nf.sample_flat(prog, f[:n2], np.random.default_rng(2))
        dt = time.perf_counter() - t0
    return {"value": n2 / dt, "unit": "shots/s", "cores": 1, "kind": "port",
            "cpu_model": cpu_model(),
            "sample": f"first {n2} shots, {dt:.1f} s: numpy sample_flat (evaluate.py:69-87) "
                      f"restated in oracle/numpy_flat.py, bit-identical to the reference's"}


def arm_config(w, shots, n_f, rng, world):
    """The config object both arms print (same workload, same keys)."""
    n_out = int(len(w.program.output_order))
    terms = sum(int(g.pf_phase_idx.shape[0]) for c in w.program.components for g in c.graphs)
    graphs = sum(len(c.graphs) for c in w.program.components)
    return {"workload": f"{w.name}: {n_out} outputs, F={n_f}, {terms} terms/shot over {graphs} graphs",
            "shots_per_gpu": shots,
            "rng": "xorshift (kokkos_sim stream)" if rng == 0 else "philox4x32-10",
            "l2": "flushed between steps (256 MiB write)",
            "parallelism": f"shot-split x{world}"}


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
            "config": arm_config(w, shots, f.shape[1], args.rng, args.gpus),
            "step_shots": step_shots,
            "cpu_baseline": {"value": value, "unit": "shots/s", "cores": threads, "kind": kind,
                             "cpu_model": cpu_model(), "sample": sample},
            "e2e": {"value": value, "unit": "shots/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _timed_launches(torch, stream, flush, fn, steps):
    """Device ms of `steps` calls of fn(i), L2 flushed before each (CUDA events)."""
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(steps)]
    for i in range(steps):
        flush.zero_()
        evs[i][0].record(stream)
        fn(i)
        evs[i][1].record(stream)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in evs]


def plain_leg(args, torch, dev, flush, cfg):
    """Another single-program workload through the plain path: device-timed
    shots/s (inputs resident, L2 flushed), the drop-in call from pinned host
    buffers, and the first rows of both outputs against the reference oracle."""
    from ksim_b200 import _abi, perfmodel, synth
    from ksim_b200.sampler import B200ProgramSampler
    L = _abi.lib()
    w = synth.config(cfg)
    shots = w.shots
    f = synth.sample_f(np.random.default_rng(w.seed + 1), shots, w.n_f, w.f_prob)
    s = B200ProgramSampler(w.program, device=dev.index or 0)
    n_out = s.num_outputs
    d_f = torch.from_numpy(f).to(dev)
    d_out = torch.zeros((shots, n_out), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def launch(seed):
        _abi.check(L.ksim_program_sample_device(
            s.handle, ctypes.c_void_p(d_f.data_ptr()), shots, w.n_f, 0, seed, args.rng,
            ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(stream.cuda_stream)))

    for i in range(max(3, args.warmup)):
        launch(100 + i)
    steps = max(3, args.steps)
    ts = _timed_launches(torch, stream, flush, lambda i: launch(200 + i), steps)
    ms = sum(ts) / len(ts)
    n_chk = min(shots, args.parity_shots if cfg != 1 else shots)
    dev_par = parity_check(w.program, f[:n_chk], d_out[:n_chk].cpu().numpy(), 200 + steps - 1, args.rng)
    f_pin = torch.from_numpy(f).pin_memory().numpy()
    out_pin = torch.empty((shots, n_out), dtype=torch.uint8).pin_memory().numpy()
    s.sample(f_pin, 300, rng_mode=args.rng, out=out_pin)
    e2e = []
    for i in range(steps):
        t0 = time.perf_counter()
        s.sample(f_pin, 400 + i, rng_mode=args.rng, out=out_pin)
        e2e.append(time.perf_counter() - t0)
    e2e_par = parity_check(w.program, f[:n_chk], out_pin[:n_chk], 400 + steps - 1, args.rng)
    work = perfmodel.program_work(w.program)
    return {"workload": arm_config(w, shots, w.n_f, args.rng, 1)["workload"], "shots": shots,
            "value": shots / (ms / 1e3), "unit": "shots/s", "ms_per_step": ms, "steps": steps,
            "e2e": {"value": shots * steps / sum(e2e), "unit": "shots/s",
                    "h2d_bytes_per_step": int(f.nbytes), "d2h_bytes_per_step": int(shots * n_out),
                    "api": "B200ProgramSampler.sample (ksim_program_sample), pinned buffers"},
            "ops_per_shot": work["ops"],
            "ops_per_shot_reference_model": perfmodel.reference_op_model(w.program),
            "parity": {"device_output": dev_par, "e2e_output": e2e_par},
            "issue_frac": (NCU_THREAD_INST_PER_SHOT[w.name] * shots / (ms / 1e3) / issue_ceiling(torch, dev)
                           if w.name in NCU_THREAD_INST_PER_SHOT else None),
            "gpu_launches": steps * len(w.program.components)}


def issue_ceiling(torch, dev, sm_mhz=None):
    """Thread instructions per second the SMs can issue: every sub-partition
    issues one warp instruction a clock (4 per SM, 32 lanes)."""
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    return sms * 4 * 32 * (sm_mhz or 1965.0) * 1e6


def bench_batched(args, torch, dev, flush):
    """Workload 3: 64 programs in one persistent graph-captured launch vs 64
    plain one-program launches on the same GPU, same inputs."""
    from ksim_b200 import synth
    from ksim_b200.batch import BatchSampler
    ws = synth.batched_workloads()
    rng = np.random.default_rng(3001)
    fs = [synth.sample_f(rng, w.shots, w.n_f, w.f_prob) for w in ws]
    seeds = [w.seed for w in ws]
    bs = BatchSampler([w.program for w in ws], [w.shots for w in ws], seeds=seeds,
                      rng_mode=args.rng, device=dev.index or 0, n_f=[w.n_f for w in ws])
    bs.set_inputs(fs)
    rec = bs.tune()
    stream = torch.cuda.current_stream(dev)
    bs.launch_plain(stream)
    plain_bits = bs.results()
    bs.launch(stream)
    same = all(np.array_equal(a, b) for a, b in zip(bs.results(), plain_bits))
    for _ in range(max(3, args.warmup)):
        bs.launch(stream)
        bs.launch_plain(stream)
    steps = max(3, args.steps)
    t_batch = _timed_launches(torch, stream, flush, lambda i: bs.launch(stream), steps)
    t_plain = _timed_launches(torch, stream, flush, lambda i: bs.launch_plain(stream), steps)
    total = bs.total_shots
    mb, mp = sum(t_batch) / steps, sum(t_plain) / steps
    info = bs.info()
    return {"workload": f"cfg3-batched: {len(ws)} programs, qubits U[8,60], t U[2,16], "
                        f"shots log-U[1e3,1e5] ({total} shots)",
            "shots_per_s": total / (mb / 1e3), "ms_per_batch": mb,
            "plain_shots_per_s": total / (mp / 1e3), "plain_ms": mp,
            "speedup_vs_plain": mp / mb, "bit_identical_to_plain": bool(same),
            "launch": "1 persistent kernel in a CUDA graph" if info["launches"] == 1
                      else f"{info['launches']} persistent kernels in a CUDA graph",
            "plain_launches": len(ws), "tuning": rec["tuning"], "work_items": info["items"],
            "grid": info["grid"],
            "issue_frac": NCU_THREAD_INST_PER_BATCH / (mb / 1e3) / issue_ceiling(torch, dev),
            "issue_note": "ncu thread instructions of one batch at the launch shape "
                          f"{NCU_BATCH_SHAPE} (this run: {rec['tuning']}) over the timed batch and "
                          "148 SMs x 4 x 32 lanes x 1965 MHz"}


class _PinnedRing:
    """FIFO allocator of output rows in one page-locked buffer (requests are
    retired in submission order)."""

    def __init__(self, torch, nbytes):
        self.buf = torch.empty(nbytes, dtype=torch.uint8).pin_memory().numpy()
        self.n = nbytes
        self.head = self.tail = 0      # byte counters (mod n)
        self.live = []                 # (start, end) in submission order
        self.cv = threading.Condition()

    def alloc(self, nbytes):
        nbytes = max(nbytes, 1)
        with self.cv:
            while True:
                pos = self.head % self.n
                skip = self.n - pos if pos + nbytes > self.n else 0   # no block across the wrap
                if self.head + skip + nbytes - self.tail <= self.n:
                    start = self.head + skip
                    self.head = start + nbytes
                    self.live.append((start, self.head))
                    s = start % self.n
                    return self.buf[s:s + nbytes]
                self.cv.wait()

    def free_oldest(self):
        with self.cv:
            self.live.pop(0)
            self.tail = self.live[0][0] if self.live else self.head
            self.cv.notify_all()


def _replay(arrivals, submit, collect):
    """Submit request i at arrivals[i] (seconds from start) on one thread and
    collect results in order on another; returns (start, done times)."""
    import queue
    q = queue.Queue()
    done = [0.0] * len(arrivals)
    t0 = time.perf_counter() + 0.05

    def producer():
        for i, a in enumerate(arrivals):
            dt = t0 + a - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            q.put((i, submit(i)))
        q.put(None)

    def consumer():
        while True:
            item = q.get()
            if item is None:
                return
            i, h = item
            done[i] = collect(i, h)

    th = [threading.Thread(target=producer), threading.Thread(target=consumer)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    return t0, done


def _batched_capacity(torch, dev, pool, pidx, shots, wide, r0, seeds, rng_mode):
    """Shots/s of requests (pool[pidx[i]], shots[i] rows of `wide` from r0[i],
    seeds[i]) run as one autotuned BatchSampler launch."""
    from ksim_b200.batch import BatchSampler
    progs = [pool[int(p)].program for p in pidx]
    nfs = [pool[int(p)].n_f for p in pidx]
    bs = BatchSampler(progs, [int(b) for b in shots], seeds=[int(s) for s in seeds], rng_mode=rng_mode,
                      device=dev.index or 0, n_f=nfs)
    bs.set_inputs([wide[int(a):int(a) + int(b), :nf] for a, b, nf in zip(r0, shots, nfs)])
    rec = bs.tune()
    stream = torch.cuda.current_stream(dev)
    for _ in range(3):
        bs.launch(stream)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    ts = _timed_launches(torch, stream, flush, lambda i: bs.launch(stream), 5)
    cap = float(np.sum(shots)) / (sum(ts) / len(ts) / 1e3)
    del bs
    return cap, rec["tuning"]


def bench_served(args, torch, dev):
    """Workload 5: a Poisson stream of sample requests over a 200-program pool
    through the continuous-batching server, and the same stream through plain
    per-request calls (B200ProgramSampler.sample) on the same GPU."""
    from ksim_b200 import synth
    from ksim_b200.sampler import B200ProgramSampler
    from ksim_b200.serve import Server
    pool = synth.serving_pool()
    rng = np.random.default_rng(5555)
    n_req = args.requests
    pidx = rng.integers(0, len(pool), n_req)
    shots = np.round(np.exp(rng.uniform(np.log(1e2), np.log(1e5), n_req))).astype(np.int64)
    rows = 100_000
    wide = torch.from_numpy(synth.sample_f(rng, rows, 128, 0.02)).pin_memory().numpy()
    r0 = (rng.random(n_req) * (rows - shots + 1)).astype(np.int64)
    seeds = rng.integers(0, 2**62, n_req)
    n_out = [p.program.num_outputs for p in pool]
    ring = _PinnedRing(torch, 1 << 30)

    srv = Server(device=dev.index or 0, arena_bytes=4 << 30, threads=args.serve_threads)
    for w in pool:                       # programs resident on the device before the stream
        d, _ = srv.cache.acquire(w.program)
        srv.cache.release(d)

    def submit(i):
        B = int(shots[i])
        out = ring.alloc(B * n_out[pidx[i]]).reshape(B, n_out[pidx[i]])
        return srv.submit(pool[pidx[i]].program, wide[r0[i]:r0[i] + B], int(seeds[i]),
                          args.rng, out=out)

    def collect(i, h):
        h.result()
        ring.free_oldest()
        return h.done_time_s

    # batched capacity of this request mix: the first requests as one
    # persistent, autotuned, graph-replayed batch (inputs resident, device time)
    n_probe = min(n_req, 1500)
    batched_capacity, batched_tuning = _batched_capacity(torch, dev, pool, pidx[:n_probe], shots[:n_probe],
                                                         wide, r0[:n_probe], seeds[:n_probe], args.rng)
    # served capacity: a closed burst of the same requests, all submitted at once
    t0, done = _replay([0.0] * n_probe, submit, collect)
    capacity = float(shots[:n_probe].sum()) / (max(done) - t0)
    rate = args.load * batched_capacity / float(shots.mean())
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_req))
    before = srv.stats()
    t0, done = _replay(arrivals, submit, collect)
    lat = np.array(done) - (t0 + arrivals)
    served = float(shots.sum()) / (max(done) - t0)
    st = srv.stats()
    srv.close()

    # the same stream through plain per-request calls, in arrival order
    samplers = {k: B200ProgramSampler(pool[k].program, device=dev.index or 0)
                for k in set(int(x) for x in pidx)}   # uploads outside the timed stream

    # page-locked outputs as the served requests get (the calls run one at a
    # time, so one buffer serves them all)
    pbuf = torch.empty(int(shots.max()) * max(n_out), dtype=torch.uint8).pin_memory().numpy()

    def pcollect(i, _):
        B = int(shots[i])
        k = int(pidx[i])
        out = pbuf[:B * n_out[k]].reshape(B, n_out[k])
        samplers[k].sample(wide[r0[i]:r0[i] + B], int(seeds[i]), rng_mode=args.rng, out=out)
        return time.perf_counter()

    pt0, pdone = _replay(arrivals, lambda i: i, pcollect)
    plat = np.array(pdone) - (pt0 + arrivals)
    plain = float(shots.sum()) / (max(pdone) - pt0)
    q = lambda a, x: float(np.percentile(a, x) * 1e3)  # noqa: E731
    return {"workload": f"cfg5-served: {n_req} Poisson requests over {len(pool)} programs "
                        f"(cfg2/3/4 generators), shots log-U[1e2,1e5], f rows 128 B",
            "shots_per_s": served, "p50_ms": q(lat, 50), "p99_ms": q(lat, 99),
            "plain_shots_per_s": plain, "plain_p50_ms": q(plat, 50), "plain_p99_ms": q(plat, 99),
            "speedup_vs_plain": served / plain,
            "arrival_rate_per_s": rate, "load": args.load,
            "load_basis": "batched capacity of the request mix (first requests as one batch)",
            "batched_capacity_shots_per_s": batched_capacity, "batched_tuning": batched_tuning,
            "served_capacity_shots_per_s": capacity,
            "total_shots": int(shots.sum()),
            "loop_launches": st["loop_launches"] - before["loop_launches"],
            "failed": st["failed"], "clock": "host wall clock, arrival -> results in host memory"}


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
    alu_peak = ctypes.c_double()
    _abi.check(L.ksim_measure_alu_peak(local, ctypes.byref(alu_peak), None))

    for i in range(args.warmup):
        launch(1000 + i)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        clk.begin()
        for i in range(args.steps):
            flush.zero_()
            evs[i][0].record(stream)
            launch(2000 + i)
            evs[i][1].record(stream)
        torch.cuda.synchronize()
        clk.end()
    barrier(world)
    torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = max_over_ranks(sum(step_ms), world)
    value = world * shots * args.steps / (total_ms / 1e3)
    ms_per_step = total_ms / args.steps
    parity = {}
    if rank == 0:
        # the last timed launch's first rows against the reference oracle
        n_chk = min(shots, args.parity_shots)
        parity["device_output"] = parity_check(prog, f[:n_chk], d_out[:n_chk].cpu().numpy(),
                                               2000 + args.steps - 1, args.rng, shot_offset=offset)

    # end to end through the drop-in API, pinned host buffers in and out
    f_pin = torch.from_numpy(f).pin_memory().numpy()
    out_pin = torch.empty((shots, n_out), dtype=torch.uint8).pin_memory().numpy()
    for i in range(max(1, args.warmup)):
        sampler.sample(f_pin, 3000 + i, rng_mode=args.rng, out=out_pin)
    barrier(world)
    e2e_t = []
    for i in range(args.steps):
        t0 = time.perf_counter()
        sampler.sample(f_pin, 4000 + i, rng_mode=args.rng, out=out_pin)
        e2e_t.append(time.perf_counter() - t0)
    e2e_total = max_over_ranks(sum(e2e_t), world)
    e2e_value = world * shots * args.steps / e2e_total
    if rank == 0:
        n_chk = min(shots, args.parity_shots)
        parity["e2e_output"] = parity_check(prog, f[:n_chk], out_pin[:n_chk], 4000 + args.steps - 1,
                                            args.rng)
    # the same through the bit-packed entry point (8 f columns / outputs per byte)
    fp_pin = torch.from_numpy(np.packbits(f, axis=1, bitorder="little")).pin_memory().numpy()
    op_pin = torch.empty((shots, (n_out + 7) // 8), dtype=torch.uint8).pin_memory().numpy()
    for i in range(max(1, args.warmup)):
        sampler.sample_packed(fp_pin, n_f, 3000 + i, rng_mode=args.rng, out=op_pin)
    barrier(world)
    e2p_t = []
    for i in range(args.steps):
        t0 = time.perf_counter()
        sampler.sample_packed(fp_pin, n_f, 4000 + i, rng_mode=args.rng, out=op_pin)
        e2p_t.append(time.perf_counter() - t0)
    e2p_value = world * shots * args.steps / max_over_ranks(sum(e2p_t), world)
    # f drawn on the device from a Pauli noise model of the workload's shape
    # (one channel per gate location), then sampled: only outputs cross PCIe
    from ksim_b200 import synth
    from ksim_b200.noise import DeviceChannelSampler
    # (the medium circuit: 40 qubits x depth 200 = 8,000 single-qubit Pauli
    # locations, X/Y/Z each p = 1e-3)
    n_loc = NOISE_LOCATIONS.get(w.name, 200)
    nprobs, nT = synth.noise_model(np.random.default_rng(w.seed + 7), n_f, n_loc)
    noise = DeviceChannelSampler(nprobs, nT, seed=w.seed, device=local)
    for i in range(max(1, args.warmup)):
        sampler.sample_noisy(noise, shots, 3000 + i, rng_mode=args.rng, out=out_pin)
    barrier(world)
    e2n_t = []
    for i in range(args.steps):
        t0 = time.perf_counter()
        sampler.sample_noisy(noise, shots, 4000 + i, noise_seed=rank * 1000 + i, rng_mode=args.rng,
                             out=out_pin)
        e2n_t.append(time.perf_counter() - t0)
    e2n_value = world * shots * args.steps / max_over_ranks(sum(e2n_t), world)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, kind, cores, n, dt = cpu_reference_rate(prog, f, 2000, args.rng, args.cpu_seconds,
                                                      shots)
        cpu = {"value": rate, "unit": "shots/s", "cores": cores, "kind": kind, "cpu_model": cpu_model(),
               "sample": f"first {n} shots of {w.name}, {dt:.1f} s on {cores} threads "
                         "(zx_eval.hpp + restated kokkos_sim loop, OpenMP)"}
    cpu_numpy = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu_numpy = numpy_baseline(prog, f, args.numpy_seconds)

    legs = {}
    if world == 1:
        for c in [int(x) for x in args.legs.split(",") if x.strip()]:
            if c != args.workload:
                legs[f"cfg{c}"] = plain_leg(args, torch, dev, flush, c)

    batched = served = None
    if world == 1 and not args.no_batched:
        batched = bench_batched(args, torch, dev, flush)
    if world == 1 and not args.no_served:
        served = bench_served(args, torch, dev)

    if rank == 0:
        mean_s = (sum(step_ms) / len(step_ms)) / 1e3
        achieved = work["ops"] * shots / mean_s
        hbm_bytes = shots * (work["in_bytes"] + work["out_bytes"])
        clocks = clk.summary()
        sm_mhz = clocks["sm_mhz"] or clocks["sm_max_mhz"] or 1965.0
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        # issue ceiling: every SM sub-partition issues one warp instruction a clock
        issue_peak = sms * 4 * 32 * sm_mhz * 1e6
        inst = NCU_THREAD_INST_PER_SHOT.get(w.name)
        issue = inst * shots / mean_s if inst else None
        ref_ops = perfmodel.reference_op_model(prog)
        roofline = {
            "bound": "issue",
            "achieved": issue / 1e12 if issue else None,
            "peak": issue_peak / 1e12,
            "unit": "T thread-instructions/s",
            "frac": issue / issue_peak if issue else None,
            "issue_frac": issue / issue_peak if issue else None,
            "inst_per_shot": inst,
            "inst_source": "ncu smsp__thread_inst_executed.sum of k_sample on this workload / shots "
                           "(one capture of 262,144 shots; summary under profiles/)",
            "peak_source": f"{sms} SMs x 4 issue slots x 32 lanes x median sampled SM clock "
                           f"({sm_mhz:.0f} MHz)",
            "ops_per_shot": work["ops"],
            "ops_per_shot_reference_model": ref_ops,
            "ops_note": "ops_per_shot: int32 operations of the formulation the kernels run; "
                        "ops_per_shot_reference_model: the reference's step-by-step algorithm "
                        "(84 per Z[w] product, 5 per 64-bit parity word); neither is an issue count",
            "int_ops_per_s": achieved,
            "int_peak_mixed": peak.value,
            "int_peak_alu": alu_peak.value,
            "ops_frac_of_mixed_peak": achieved / peak.value,
            "ops_frac_of_alu_peak": achieved / alu_peak.value,
            "reference_model_ops_per_s": ref_ops * shots / mean_s,
            "traffic": (NCU_DRAM_BYTES_PER_SHOT[w.name] * shots
                        if w.name in NCU_DRAM_BYTES_PER_SHOT else None),
            "traffic_unit": "bytes per launch",
            "algorithmic_bytes": hbm_bytes,
            "hbm_gbs": hbm_bytes / mean_s / 1e9,
        }
        line = {
            "metric": METRIC, "value": value, "unit": "shots/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic",
            "config": arm_config(w, shots, n_f, args.rng, world),
            "e2e": {"value": e2e_value, "unit": "shots/s", "h2d_bytes_per_step": int(f.nbytes),
                    "d2h_bytes_per_step": int(shots * n_out),
                    "api": "B200ProgramSampler.sample (ksim_program_sample), pinned buffers"},
            "e2e_noisy": {"value": e2n_value, "unit": "shots/s", "h2d_bytes_per_step": 0,
                          "d2h_bytes_per_step": int(shots * n_out),
                          "api": "B200ProgramSampler.sample_noisy (ksim_program_sample_noisy): "
                                 f"f drawn on the device from {n_loc} Pauli channels "
                                 f"({noise.num_channels} after merging)"},
            "e2e_packed": {"value": e2p_value, "unit": "shots/s",
                           "h2d_bytes_per_step": int(fp_pin.nbytes),
                           "d2h_bytes_per_step": int(shots * ((n_out + 7) // 8)),
                           "api": "B200ProgramSampler.sample_packed (ksim_program_sample_packed)"},
            "roofline": roofline,
            "parity": parity,
            "cpu_baseline": cpu,
            "cpu_baseline_numpy": cpu_numpy,
            "legs": legs,
            "batched": batched,
            "served": served,
            "clocks": clocks,
            "gpu_launches": args.steps * len(prog.components),
            "step_ms": step_ms,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
