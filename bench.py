#!/usr/bin/env python3
"""Converged steady cases per second and p50/p99 time-to-converge of the batched service.

Workload: the batched 2D lid-driven-cavity sweep -- cases with mesh edge n drawn log-uniform
from 16 to 256 (256 to 65,536 cells) and Re uniform in 50..1000, seeded (seed 2024 gives the
512-case sweep; the stream continues with seeds 2025, 2026, ... in blocks of 512), steady
SIMPLE (urf U 0.7, p 0.3, two p correctors), converged to scaled residuals <= 1e-6. The service
keeps up to --budget cells resident per GPU (continuous batching: a case is admitted as soon as
cells free up), advances every resident case by one SIMPLE iteration per tick (U: FP64
multicolour Gauss-Seidel; p: FP32 agglomeration-AMG V-cycle preconditioning FP64 flexible CG),
and replays each tick as one CUDA graph.

A step is --ticks service ticks. `value` counts the cases that converged during the K timed
steps, over the device time of those steps (CUDA events on the service's stream, which carry
the admissions of new cases too; results stay on the device). `e2e` repeats the measurement
through the public API from host buffers: cases are submitted from host arrays inside the
timed region, and each converged case's U and p are read back to host and released.

Beside it the line carries: the roofline of the dominant kernel (measured live on the resident
batch), the CPU baseline (the C++ oracle, a serial restatement of the reference's algorithm,
timed per SIMPLE iteration on host cores and applied to the sweep's iteration counts), and the
plain FP64 one-case-at-a-time GPU form timed the same way.

Multi-GPU: one process per GPU; case i of the stream goes to rank i mod N (independent cases,
no data-path collective; weak scaling). Timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SWEEP = 512
SEED0 = 2024
ITER_FIXTURE = os.path.join(ROOT, "tests", "golden", "c4_sweep_iterations.json")


def parse():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=16)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--ticks", type=int, default=25, help="service ticks per step")
    ap.add_argument("--budget", type=int, default=8_000_000, help="resident cells per GPU")
    ap.add_argument("--admit-interval", type=int, default=8, help="service steps between admissions")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-workers", type=int, default=0, help="0: all host cores (at most 64)")
    ap.add_argument("--profile-plain", choices=("C1", "C2", "C3"), default=None,
                    help="profiling run for ncu: one plain FP64 SIMPLE iteration of a named single-case "
                         "workload inside cudaProfilerStart/Stop (after one warm-up iteration)")
    ap.add_argument("--workload", choices=("sweep", "serving"), default="sweep",
                    help="sweep: the 2D cavity sweep stream (the headline line); serving: the Poisson-arrival mix "
                         "of 2D/3D cavities and tet channels (its own JSON line)")
    ap.add_argument("--serving-requests", type=int, default=48, help="requests per serving phase")
    ap.add_argument("--capacity-steps", type=int, default=400, help="service steps of the closed-loop phase")
    ap.add_argument("--plain-kernels", action="store_true",
                    help="only the plain FP64 form's solver-kernel rooflines on the 1M-cell tet channel (one JSON "
                         "line per kernel; the ncu target for those kernels)")
    ap.add_argument("--profile", action="store_true",
                    help="profiling run for ncu: eager launches, warm-up only, then one roofline unit of the "
                         "dominant kernel and one step inside cudaProfilerStart/Stop; prints the unit's bytes")
    return ap.parse_args()


# ------------------------------------------------------------------ workload
def stream_params(i: int):
    from matlab_ufvm_b200 import case
    b = i // SWEEP
    key = (b,)
    if key not in _PARAM_CACHE:
        _PARAM_CACHE[key] = case.batched_sweep_params(SWEEP, seed=SEED0 + b)
    return _PARAM_CACHE[key][i % SWEEP]


_PARAM_CACHE: dict = {}
_SPEC_CACHE: dict = {}


def base_spec(n: int):
    from matlab_ufvm_b200 import case
    if n not in _SPEC_CACHE:
        _SPEC_CACHE[n] = case.cavity_case(n, nu=0.01, quirks=case.QUIRKS_CONVERGING)
    return _SPEC_CACHE[n]


def case_spec(i: int):
    import dataclasses
    n, re = stream_params(i)
    return dataclasses.replace(base_spec(n), nu=1.0 / re, name=f"sweep{i}_n{n}_Re{re:.0f}")


def _mesh_worker(n):
    from matlab_ufvm_b200 import case
    return n, case.cavity_case(n, nu=0.01, quirks=case.QUIRKS_CONVERGING)


def prebuild_meshes(indices, ranks: int = 1):
    """Builds the cavity meshes the run needs in a spawn pool, sharing the host cores with the
    other ranks of the node."""
    import multiprocessing as mp
    need = sorted({stream_params(i)[0] for i in indices} - set(_SPEC_CACHE))
    if not need:
        return
    procs = max(1, min(len(need), (os.cpu_count() or 2) // max(1, ranks) - 1, 32))
    if procs == 1 or len(need) < 4:
        for n in need:
            base_spec(n)
        return
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        for n, spec in pool.imap_unordered(_mesh_worker, sorted(need, reverse=True)):
            _SPEC_CACHE[n] = spec


def mesh_bytes(spec) -> int:
    m = spec.mesh
    return int(m.points.nbytes + m.face_start.nbytes + m.face_nodes.nbytes + m.owner.nbytes + m.neighbour.nbytes
               + spec.val_u.nbytes + spec.val_p.nbytes + 8 * len(m.patches) * 4)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ distributed plumbing
def dist_setup(args):
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, ws, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def reduce_max(x: float, ws: int) -> float:
    from matlab_ufvm_b200 import sharding
    return sharding.reduce_max(x)


def reduce_sum(x: float, ws: int) -> float:
    from matlab_ufvm_b200 import sharding
    return sharding.reduce_sum(x)


def gather_list(xs, ws):
    from matlab_ufvm_b200 import sharding
    return sharding.gather(xs)


# ------------------------------------------------------------------ the service run
class Feeder:
    """Keeps the service's queue filled from this rank's share of the case stream."""

    def __init__(self, svc, rank, ws, max_iter=20000, depth=256):
        self.svc, self.rank, self.ws, self.max_iter, self.depth = svc, rank, ws, max_iter, depth
        self.k = 0
        self.queued = 0
        self.tickets = []
        self.h2d = 0

    def next_index(self):
        from matlab_ufvm_b200 import sharding
        i = sharding.stream_index(self.rank, self.ws, self.k)
        self.k += 1
        return i

    def fill(self, n_queued):
        while n_queued < self.depth:
            spec = case_spec(self.next_index())
            self.tickets.append(self.svc.submit(spec, self.max_iter))
            self.h2d += mesh_bytes(spec)
            n_queued += 1


def run_service(args, rank, ws, e2e: bool):
    import torch
    from matlab_ufvm_b200 import ufvm
    settings = ufvm.fast_settings(base_spec(16))
    svc = ufvm.Service(settings, max_resident_cells=args.budget)
    svc.set_admit_interval(args.admit_interval)
    stream = torch.cuda.ExternalStream(svc.stream())
    feed = Feeder(svc, rank, ws)
    feed.fill(0)
    state = {"nr": 0, "nq": feed.depth, "d2h": 0}
    finished = []  # (ticket, status dict) in completion order

    def tick():
        nr, nq, nf = svc.step()
        state["d2h"] += nr * (24 * 8 + 4 * 4 + 16)  # per-step residual scalars and flags read back
        for t in svc.poll():
            st = svc.status(t)
            if e2e:
                # read the result back to host memory through the public API and free the slot
                if st["state"] == "converged":
                    state["d2h"] += svc.field(t, "U").nbytes + svc.field(t, "p").nbytes
                svc.release(t)
            finished.append((t, st))
        feed.fill(nq)

    for _ in range(args.warmup * args.ticks):
        tick()
    n_before = len(finished)
    s0 = svc.stats()
    h2d0, d2h0 = feed.h2d, state["d2h"]
    torch.cuda.synchronize()
    barrier(ws)
    clk = ClockSampler(torch.cuda.current_device()) if rank == 0 and not e2e else None
    if clk:
        clk.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    w0 = time.perf_counter()
    for _ in range(args.steps * args.ticks):
        tick()
    ev1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    ms = ev0.elapsed_time(ev1)
    barrier(ws)
    clocks = clk.stop() if clk else None
    s1 = svc.stats()
    win = [st for _, st in finished[n_before:] if st["state"] == "converged"]
    out = dict(ms=ms, wall=wall, converged=len(win), ttc=[st["latency_ms"] for st in win],
               queue=[st["queue_ms"] for st in win], iters=[st["iterations"] for st in win],
               stopped=sum(1 for _, st in finished[n_before:] if st["state"] != "converged"),
               launches=s1["graph_launches"] - s0["graph_launches"],
               graph_ticks=s1["graph_ticks"] - s0["graph_ticks"], ticks=s1["steps"] - s0["steps"],
               captures=s1["captures"] - s0["captures"],
               h2d=feed.h2d - h2d0, d2h=state["d2h"] - d2h0, clocks=clocks)
    return svc, out


ROOF_KERNEL = (1, "k_mc32_l0 (FP32 multicolour Gauss-Seidel sweep of the V-cycle's level 0, "
                  "colour-permuted ELL; one unit = both colours forward then backward over every case)")


def main_profile(args):
    """ncu target: the kernels of one unit of the roofline kernel and of one eager step."""
    import torch
    from matlab_ufvm_b200 import build as _b, ufvm
    torch.cuda.set_device(0)
    _b.build()
    # meshes are built on demand in this process (no worker pool under the profiler)
    settings = ufvm.fast_settings(base_spec(16))
    settings.service_eager = 1
    svc = ufvm.Service(settings, max_resident_cells=args.budget)
    svc.set_schedule(8192)
    feed = Feeder(svc, 0, 1)
    feed.fill(0)
    for _ in range(args.warmup * args.ticks):
        nr, nq, nf = svc.step()
        svc.poll()
        feed.fill(nq)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    ms, by = svc.profile(ROOF_KERNEL[0], 1)
    svc.step()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"profile_unit_bytes": by, "profile_unit_ms": ms, "resident": nr}), flush=True)
    svc.close()
    return 0


def main_profile_plain(args):
    """ncu target: one iteration of the plain FP64 form on a named workload."""
    import torch
    from matlab_ufvm_b200 import build as _b, case, ufvm
    torch.cuda.set_device(0)
    _b.build()
    make = {"C1": lambda: case.cavity_case(20, nu=0.01),
            "C2": lambda: case.cavity_case(64, nu=1.0 / 400, dim=3, p_smoother="ILU"),
            "C3": lambda: case.channel_case()}[args.profile_plain]
    g = ufvm.GpuCase(make())
    g.iterate()
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    t0 = time.perf_counter()
    g.iterate()
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    torch.cuda.profiler.stop()
    print(json.dumps({"plain_iteration_s": el, "workload": args.profile_plain}), flush=True)
    g.close()
    return 0


def roofline(svc, peaks):
    """Dominant kernel, timed live on the resident batch."""
    kernel_id, name = ROOF_KERNEL
    ms, by = svc.profile(kernel_id, 20)
    achieved = by / (ms * 1e-3) / 1e9
    peak = peaks.get("hbm_gbs")
    others = []
    for kid, kname in ((0, "k_mc64 (FP64 multicolour Gauss-Seidel sweep of U, ELL copy)"),
                       (2, "k_fcg_q (FP64 q = A p with (p, q) and (p, r))")):
        m2, b2 = svc.profile(kid, 20)
        a2 = b2 / (m2 * 1e-3) / 1e9
        others.append({"kernel": kname, "achieved": round(a2, 1), "frac": round(a2 / peak, 4) if peak else None,
                       "bytes_per_unit": b2, "ms_per_unit": round(m2, 4)})
    return {"kernel": name, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4) if peak else None, "traffic": None,
            "bytes_per_unit": by, "ms_per_unit": round(ms, 4),
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peak else "unavailable (fallback)",
            "other_kernels": others}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    out = {}
    if os.path.exists(p):
        try:
            d = json.load(open(p))
            for k in ("hbm_gbs", "bf16_tflops"):
                v = d.get(k)
                if isinstance(v, dict):
                    v = v.get("value")
                if isinstance(v, (int, float)):
                    out[k] = float(v)
        except (ValueError, OSError):
            pass
    if "hbm_gbs" not in out:
        out["hbm_gbs"] = 6650.0
        out["fallback"] = True
    return out


# ------------------------------------------------------------------ per-iteration cost models
SAMPLE_N = (16, 24, 32, 48, 64, 96, 128, 192, 256)


def sweep_iterations():
    """Iterations to converge of the 512 sweep cases (service, same SIMPLE settings)."""
    d = json.load(open(ITER_FIXTURE))
    return [(int(c["n"]), int(c["iterations"])) for c in d["cases"]]


def interp_cost(samples: dict, n: int) -> float:
    """log-log interpolation of seconds per iteration over the sampled sizes."""
    xs = sorted(samples)
    if n <= xs[0]:
        return samples[xs[0]] * (n / xs[0]) ** 2
    if n >= xs[-1]:
        return samples[xs[-1]] * (n / xs[-1]) ** 2
    for a, b in zip(xs, xs[1:]):
        if a <= n <= b:
            la, lb = math.log(samples[a]), math.log(samples[b])
            f = (math.log(n) - math.log(a)) / (math.log(b) - math.log(a))
            return math.exp(la + f * (lb - la))
    return samples[xs[-1]]


def _oracle_sample(arg):
    """Seconds per SIMPLE iteration of the oracle (one core) on a cavity of edge n."""
    n, budget_s = arg
    from matlab_ufvm_b200 import case
    from oracle import oracle
    spec = case.cavity_case(n, nu=1.0 / 500.0, quirks=case.QUIRKS_CONVERGING)
    oc = oracle.OracleCase(spec)
    oc.iterate()  # warm-up
    t0 = time.perf_counter()
    k = 0
    while True:
        oc.iterate()
        k += 1
        el = time.perf_counter() - t0
        if el > budget_s or k >= 20:
            break
    return n, el / k, k


def cpu_baseline(workers: int, budget_s: float):
    """Oracle cost per iteration at the sample sizes, all workers busy at once (spawn pool)."""
    import multiprocessing as mp
    from oracle import oracle
    oracle.build()
    ctx = mp.get_context("spawn")
    jobs = [(n, budget_s) for n in SAMPLE_N]
    jobs = (jobs * ((workers + len(jobs) - 1) // len(jobs)))[:max(workers, len(jobs))]
    t0 = time.perf_counter()
    with ctx.Pool(workers) as pool:
        res = pool.map(_oracle_sample, jobs)
    wall = time.perf_counter() - t0
    per = {}
    for n, s, k in res:
        per.setdefault(n, []).append(s)
    samples = {n: statistics.median(v) for n, v in per.items()}
    its = sweep_iterations()
    seconds_per_case = statistics.mean(it * interp_cost(samples, n) for n, it in its)
    return {"cases_per_s": workers / seconds_per_case, "s_per_iter": samples, "wall": wall,
            "seconds_per_case": seconds_per_case}


def plain_gpu_sample(budget_s: float):
    """The plain FP64 form (reference smoothers, AMG rebuilt every p solve) one case at a time."""
    import torch
    from matlab_ufvm_b200 import case, ufvm
    samples = {}
    for n in (16, 32, 64, 128, 256):
        spec = case.cavity_case(n, nu=1.0 / 500.0, quirks=case.QUIRKS_CONVERGING)
        g = ufvm.GpuCase(spec)
        g.iterate()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        k = 0
        while True:
            g.iterate()
            k += 1
            if time.perf_counter() - t0 > budget_s / 5 or k >= 10:
                break
        torch.cuda.synchronize()
        samples[n] = (time.perf_counter() - t0) / k
        g.close()
    its = sweep_iterations()
    seconds_per_case = statistics.mean(it * interp_cost(samples, n) for n, it in its)
    return {"cases_per_s": 1.0 / seconds_per_case, "s_per_iter": samples, "seconds_per_case": seconds_per_case}


def plain_kernel_rooflines(peaks):
    """The plain FP64 form's solver kernels on the 1,029,000-cell tet channel's momentum matrix
    (device arrays), kernel time only: the library's profiling entry point prepares schedules,
    colourings and the DILU factor, then times each launch with CUDA events after a read of
    twice the L2 size."""
    import torch
    from matlab_ufvm_b200 import case, ufvm
    spec = case.channel_case()
    g = ufvm.GpuCase(spec)
    g.iterate()
    g.cfdUpdateFields()
    g.cfdAssembleEquation("U", 1)
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda()
           for a in (g.level_array(0, "rowptr"), g.level_array(0, "col"), g.get("ac"), g.get("anb"), g.get("bc"))]
    g.close()
    n, nnz = dev[2].numel(), dev[3].numel()
    out = []
    for key, name in (
            ("residual", "k_residual (plain FP64 r = b - A x, cfdComputeResidualsArray)"),
            ("MCGS", "k_mc_rows (plain FP64 symmetric multicolour Gauss-Seidel, colour-major ELL copy)"),
            ("SOR", "k_sched_sell (plain FP64 symmetric natural-order Gauss-Seidel, level scheduled, "
                    "cfdSolveSOR: latency-bound by its dependency levels)"),
            ("ILU", "k_ilu_res + k_sched_sell (plain FP64 DILU application, level scheduled, cfdSolveILU: "
                    "latency-bound by its dependency levels)")):
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        ms, by = ufvm.profile_plain_kernel(key, *dev, x, 5)
        a = by / (ms * 1e-3) / 1e9
        out.append({"kernel": name, "rows": n, "nnz": nnz, "bytes": by, "ms": round(ms, 4),
                    "achieved": round(a, 1), "unit": "GB/s",
                    "frac": round(a / peaks["hbm_gbs"], 4) if peaks.get("hbm_gbs") else None})
    return out


def plain_named_configs():
    """Seconds per steady SIMPLE iteration of the plain FP64 form on the named single-case
    workloads, on the GPU and in the oracle (one host core), same settings as the reference's
    tutorials: the 20x20 cavity (Re 100), the 64^3 cavity (Re 400, ILU for p) and the
    1,029,000-cell jittered-tet channel (Re 200)."""
    import torch
    from matlab_ufvm_b200 import case, ufvm
    from oracle import oracle
    oracle.build()
    out = {}
    for key, make, n_gpu, n_cpu in (
            ("C1_cavity_20x20", lambda: case.cavity_case(20, nu=0.01), 10, 10),
            ("C2_cavity_64cubed_ilu", lambda: case.cavity_case(64, nu=1.0 / 400, dim=3, p_smoother="ILU"), 4, 2),
            ("C3_channel_1M_tet", lambda: case.channel_case(), 3, 1)):
        spec = make()
        g = ufvm.GpuCase(spec)
        g.iterate()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(n_gpu):
            g.iterate()
        torch.cuda.synchronize()
        gpu = (time.perf_counter() - t0) / n_gpu
        g.close()
        oc = oracle.OracleCase(spec)
        oc.iterate()
        t0 = time.perf_counter()
        for _ in range(n_cpu):
            oc.iterate()
        cpu = (time.perf_counter() - t0) / n_cpu
        del oc
        out[key] = {"cells": spec.mesh.n_cells, "gpu_ms_per_iteration": round(gpu * 1e3, 3),
                    "oracle_ms_per_iteration": round(cpu * 1e3, 3), "oracle_cores": 1,
                    "speedup": round(cpu / gpu, 2)}
    return out


def pct(v, q):
    return float(np.percentile(np.asarray(v), q)) if len(v) else None


# ------------------------------------------------------------------ arms
def main_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    workers = args.cpu_workers or min(os.cpu_count() or 1, 64)
    budget = 2.0
    for _ in range(args.warmup):
        cpu_baseline(workers, 0.3)
    vals = []
    last = None
    t0 = time.perf_counter()
    for _ in range(args.steps):
        last = cpu_baseline(workers, budget)
        vals.append(last["cases_per_s"])
    el = time.perf_counter() - t0
    v = statistics.median(vals)
    line = {
        "impl": "reference", "metric": "converged_cases_per_s", "value": v, "unit": "cases/s",
        "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args),
        "cpu_baseline": {"value": v, "unit": "cases/s", "cores": workers, "kind": "port",
                         "sample": f"C++ oracle (serial restatement of the reference SIMPLE/AMG loop), "
                                   f"seconds per SIMPLE iteration at n in {list(SAMPLE_N)} "
                                   f"(Re 500) on {workers} concurrent processes, applied to the 512 sweep "
                                   f"cases' iteration counts; {workers} cases in parallel"},
        "e2e": {"value": v, "unit": "cases/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "s_per_iter": {str(k): round(s, 6) for k, s in last["s_per_iter"].items()},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(args):
    return {"workload": "2D lid-driven cavity sweep stream: n log-uniform 16..256, Re uniform 50..1000, "
                        "seeds 2024+ (first 512 = the batched sweep), SIMPLE to scaled residual 1e-6",
            "resident_cells_per_gpu": args.budget, "ticks_per_step": args.ticks,
            "l2": "inputs larger than L2 (resident batch of up to ~6M cells, GBs of matrices and fields)",
            "parallelism": f"case-sharded x{args.gpus}"}


def main_ours(args):
    import torch
    rank, ws, local = dist_setup(args) if args.gpus > 1 or int(os.environ.get("WORLD_SIZE", "1")) > 1 \
        else (0, 1, 0)
    if not torch.cuda.is_available():
        print(json.dumps({"error": "no CUDA device"}), flush=True)
        return 1
    if ws == 1:
        torch.cuda.set_device(0)
    from matlab_ufvm_b200 import build as _b
    _b.build()
    # meshes for the first cases of this rank's share (the rest are built on demand)
    from matlab_ufvm_b200 import sharding
    prebuild_meshes([sharding.stream_index(rank, ws, k) for k in range(1200 // ws + 1)], ws)
    peaks = load_peaks()
    svc, res = run_service(args, rank, ws, e2e=False)
    roof = roofline(svc, peaks) if rank == 0 else None
    svc.close()
    total = reduce_sum(res["converged"], ws)
    ms = reduce_max(res["ms"], ws)
    value = total / (ms * 1e-3) if ms > 0 else 0.0
    ttc = gather_list(res["ttc"], ws)
    qms = gather_list(res["queue"], ws)
    e2e = None
    if not args.no_e2e:
        svc2, r2 = run_service(args, rank, ws, e2e=True)
        svc2.close()
        tot2 = reduce_sum(r2["converged"], ws)
        ms2 = reduce_max(r2["ms"], ws)
        e2e = {"value": tot2 / (ms2 * 1e-3) if ms2 > 0 else 0.0, "unit": "cases/s",
               "h2d_bytes_per_step": int(reduce_sum(r2["h2d"], ws) / args.steps),
               "d2h_bytes_per_step": int(reduce_sum(r2["d2h"], ws) / args.steps),
               "wall_s": round(r2["wall"], 3)}
    plain = cpu = None
    if rank == 0 and ws == 1:
        if not args.no_plain:
            plain = plain_gpu_sample(20.0)
            plain["kernels"] = plain_kernel_rooflines(peaks)
            plain["named"] = plain_named_configs()
        if not args.no_cpu:
            workers = args.cpu_workers or min(os.cpu_count() or 1, 64)
            cpu = cpu_baseline(workers, 2.0)
    launches = int(reduce_sum(res["launches"], ws))
    if rank == 0:
        line = {
            "metric": "converged_cases_per_s", "value": value, "unit": "cases/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
            "data": "synthetic (seeded cavity meshes generated in-process)",
            "config": workload_config(args),
            "time_to_converge_ms": {"p50": pct(ttc, 50), "p99": pct(ttc, 99), "n": len(ttc),
                                    "clock": "service device clock, admission to convergence"},
            "queue_ms": {"p50": pct(qms, 50), "p99": pct(qms, 99)},
            "converged_in_window": int(total), "stopped_in_window": int(reduce_sum(res["stopped"], ws)),
            "ticks_timed": res["ticks"], "graph_ticks": res["graph_ticks"], "graph_captures": res["captures"],
            "roofline": roof, "e2e": e2e, "gpu_launches": launches, "clocks": res["clocks"],
        }
        if cpu:
            line["cpu_baseline"] = {
                "value": cpu["cases_per_s"], "unit": "cases/s", "cores": args.cpu_workers or min(os.cpu_count() or 1, 64),
                "kind": "port",
                "sample": "C++ oracle seconds per SIMPLE iteration at n in %s (Re 500, 2 s each), applied to the "
                          "512 sweep cases' iteration counts" % (list(SAMPLE_N),),
                "s_per_iter": {str(k): round(s, 6) for k, s in cpu["s_per_iter"].items()}}
        if plain:
            line["plain_fp64_gpu"] = {
                "value": plain["cases_per_s"], "unit": "cases/s",
                "method": "plain FP64 form (reference SOR/ILU smoothers, AMG rebuilt every p solve) one case at a "
                          "time: seconds per SIMPLE iteration at n in 16..256 applied to the sweep's iteration counts",
                "s_per_iter": {str(k): round(s, 6) for k, s in plain["s_per_iter"].items()},
                "kernels_1M_tet_channel": plain["kernels"], "named_configs": plain["named"]}
            line["batched_over_plain"] = value / plain["cases_per_s"] if plain["cases_per_s"] else None
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def _serving_worker(key):
    from matlab_ufvm_b200 import serving
    kind, size = key
    return key, serving.request_spec(serving.Request(0, kind, size, 100.0))


def main_serving(args):
    """The serving mix on one GPU: 70% 2D cavities of 1k-64k cells, 25% 3D cavities 32^3-96^3,
    5% tet channels of 0.5-2M cells, Re 50..1000. A closed-loop phase (queue kept full) measures
    the capacity in converged cases per second of service clock; an open-loop phase on a fresh
    service then submits a second seeded stream at Poisson arrival times of 0.8 x that rate and
    reports throughput and time-to-converge percentiles from arrival."""
    import dataclasses
    import multiprocessing as mp
    import torch
    from matlab_ufvm_b200 import build as _b, serving, ufvm
    torch.cuda.set_device(0)
    _b.build()
    cap_reqs = serving.serving_mix(args.serving_requests, seed=101)
    open_reqs = serving.serving_mix(args.serving_requests, seed=202)
    keys = sorted({(r.kind, r.size) for r in cap_reqs + open_reqs}, key=lambda k: -serving.Request(0, *k, 1.0).cells)
    base = {}
    procs = max(1, min(len(keys), (os.cpu_count() or 2) - 1, 16))
    with mp.get_context("spawn").Pool(procs) as pool:
        for key, spec in pool.imap_unordered(_serving_worker, keys):
            base[key] = spec

    def spec_fn(req):
        return dataclasses.replace(base[(req.kind, req.size)], nu=1.0 / req.re, name=f"serving{req.index}")

    settings = ufvm.fast_settings(base_spec(16))

    def service():
        svc = ufvm.Service(settings, max_resident_cells=args.budget)
        svc.set_admit_interval(args.admit_interval)
        return svc

    svc = service()
    cap = serving.closed_loop_capacity(svc, cap_reqs, args.capacity_steps, spec_fn=spec_fn)
    svc.close()
    rate = 0.8 * cap["cases_per_s"]
    line = {"workload": "serving mix (70% 2D cavities 1k-64k cells, 25% 3D cavities 32^3-96^3, 5% tet channels "
                        "0.5-2M cells, Re 50..1000, seeded)", "n_gpus": 1, "budget_cells": args.budget,
            "capacity": cap, "arrival_rate_per_s": rate}
    if rate > 0:
        svc = service()
        arr = serving.poisson_arrivals(len(open_reqs), rate, seed=303)
        ol = serving.OpenLoop(svc, open_reqs, arr, spec_fn=spec_fn)
        out = ol.run()
        svc.close()
        line.update(metric="converged cases/s + p50/p99 time to converge (from arrival, service clock)",
                    open_loop=serving.summarize(out), service_steps=ol.steps, idle_s=ol.idle_s)
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return main_reference(args)
    if args.profile:
        return main_profile(args)
    if args.profile_plain:
        return main_profile_plain(args)
    if args.workload == "serving":
        return main_serving(args)
    if args.plain_kernels:
        import torch
        from matlab_ufvm_b200 import build as _b
        torch.cuda.set_device(0)
        _b.build()
        for row in plain_kernel_rooflines(load_peaks()):
            print(json.dumps(row), flush=True)
        return 0
    return main_ours(args)


if __name__ == "__main__":
    sys.exit(main())
