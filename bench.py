#!/usr/bin/env python3
"""Converged steady cases per second and p50/p99 time-to-converge of the batched service.

Workload (the batched-sweep configuration): 512 independent 2D lid-driven cavities, mesh edge n
drawn log-uniform from 16 to 256 (256 to 65,536 cells) and Re uniform in 50..1000 (seed 2024),
steady SIMPLE (urf U 0.7, p 0.3, two p correctors), each converged to scaled residuals <= 1e-6.
All 512 are resident together (about 5.7M cells); every tick advances each unfinished case by
one SIMPLE iteration (U: FP64 multicolour Gauss-Seidel; p: FP32 agglomeration-AMG V-cycle
preconditioning FP64 flexible CG) and is replayed as one CUDA graph.

Timing: a step is --ticks service ticks and the K timed steps cover the whole batch (its slowest
case needs about 3,500 iterations; the default is 20 steps of 200 ticks), so every case converges
inside the timed region: `value` = converged cases / device time of the K steps (CUDA events on
the service's stream). The meshes are uploaded and processed (admission) before the timed region.
`e2e` repeats the batch through the public API from host buffers: submission from host arrays,
admission (host-to-device copies), all ticks, and the read-back of every converged case's U and p
to host memory, timed on the host clock.

Warm-up: W steps of the same length on a second 512-case batch of the same distribution (seed
1999). While that batch is resident (inputs larger than L2), the roofline kernels are timed on it.

Beside the line: the reference arm (`--impl reference`: the C++ oracle, a serial restatement of the
reference's algorithm, on every host core), the same CPU measurement as `cpu_baseline`, and the
plain FP64 one-case-at-a-time GPU form.

Multi-GPU: one process per GPU; rank r solves its own 512-case batch (seed 2024 + r): weak scaling,
no data-path collective. The timed duration is the max over ranks.
"""
from __future__ import annotations

import argparse
import dataclasses
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
WARM_SEED = 1999
ORACLE_FIXTURE = os.path.join(ROOT, "tests", "golden", "sweep_oracle.json")
PLAIN_FIXTURE = os.path.join(ROOT, "tests", "golden", "sweep_oracle_plain.json")
PLAIN_SETTINGS = {"p_smoother": "MCGS"}  # the plain form: V-cycle + multicolour GS for p, DILU for U


def parse():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--ticks", type=int, default=200, help="service ticks per step")
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
                    help="sweep: the 512-case 2D cavity batch (the headline line); serving: the Poisson-arrival "
                         "mix of 2D/3D cavities and tet channels (its own JSON line)")
    ap.add_argument("--serving-requests", type=int, default=96, help="requests per serving phase")
    ap.add_argument("--capacity-steps", type=int, default=400, help="service steps of the closed-loop phase")
    ap.add_argument("--serving-max-iter", type=int, default=8000,
                    help="SIMPLE iteration limit of a serving request (the case script's endTime)")
    ap.add_argument("--plain-kernels", action="store_true",
                    help="only the plain FP64 form's solver-kernel rooflines on the 1M-cell tet channel (one JSON "
                         "line per kernel; the ncu target for those kernels)")
    ap.add_argument("--profile", action="store_true",
                    help="profiling run for ncu: eager launches, warm-up only, then one roofline unit of the "
                         "dominant kernel and one step inside cudaProfilerStart/Stop; prints the unit's bytes")
    ap.add_argument("--profile-cases", type=int, default=128, help="cases resident in the --profile run")
    return ap.parse_args()


# ------------------------------------------------------------------ workload
_SPEC_CACHE: dict = {}


def base_spec(n: int):
    from matlab_ufvm_b200 import case
    if n not in _SPEC_CACHE:
        _SPEC_CACHE[n] = case.cavity_case(n, nu=0.01, quirks=case.QUIRKS_CONVERGING)
    return _SPEC_CACHE[n]


def batch_params(seed: int, count: int = SWEEP):
    from matlab_ufvm_b200 import case
    return case.batched_sweep_params(count, seed=seed)


def batch_specs(seed: int, count: int = SWEEP):
    return [dataclasses.replace(base_spec(n), nu=1.0 / re, name=f"sweep{seed}_{i}_n{n}_Re{re:.0f}")
            for i, (n, re) in enumerate(batch_params(seed, count))]


def _mesh_worker(n):
    from matlab_ufvm_b200 import case
    return n, case.cavity_case(n, nu=0.01, quirks=case.QUIRKS_CONVERGING)


def prebuild_meshes(sizes, ranks: int = 1):
    """Builds the cavity meshes the run needs in a spawn pool, sharing the host cores with the
    other ranks of the node."""
    import multiprocessing as mp
    need = sorted(set(sizes) - set(_SPEC_CACHE))
    if not need:
        return
    procs = max(1, min(len(need), (os.cpu_count() or 2) // max(1, ranks) - 1, 32))
    if procs == 1 or len(need) < 4:
        for n in need:
            base_spec(n)
        return
    with mp.get_context("spawn").Pool(procs) as pool:
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


# ------------------------------------------------------------------ the service runs
MAX_ITER = 20000
STEP_D2H = 24 * 8 + 4 * 4 + 16  # per resident case and tick: residual scalars and flags read back


def service_settings():
    from matlab_ufvm_b200 import ufvm
    return ufvm.fast_settings(base_spec(16))


def new_service(args):
    from matlab_ufvm_b200 import ufvm
    svc = ufvm.Service(service_settings(), max_resident_cells=args.budget)
    svc.set_admit_interval(args.admit_interval)
    return svc


def warm_up(args):
    """W steps on the warm-up batch; returns the service with that batch still resident."""
    import torch
    svc = new_service(args)
    for s in batch_specs(WARM_SEED):
        svc.submit(s, MAX_ITER)
    svc.admit()
    for _ in range(args.warmup * args.ticks):
        nr, nq, _ = svc.step()
        for t in svc.poll():
            svc.release(t)
        if nr == 0 and nq == 0:
            break
    torch.cuda.synchronize()
    return svc


def run_batch(args, specs, ws, e2e: bool, rank: int, keep=()):
    """The timed batch: every case of `specs` to convergence in K steps of --ticks ticks. In the
    e2e pass, the read-back U and p of the cases whose positions are in `keep` are returned too."""
    import torch
    svc = new_service(args)
    stream = torch.cuda.ExternalStream(svc.stream())
    h2d = d2h = 0
    tickets = []
    admit_s = None
    if not e2e:
        tickets = [svc.submit(s, MAX_ITER) for s in specs]
        torch.cuda.synchronize()
        a0 = time.perf_counter()
        svc.admit()
        torch.cuda.synchronize()
        admit_s = time.perf_counter() - a0
    torch.cuda.synchronize()
    barrier(ws)
    clk = ClockSampler(torch.cuda.current_device()) if rank == 0 and not e2e else None
    if clk:
        clk.start()
    s0 = svc.stats()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    w0 = time.perf_counter()
    if e2e:
        for s in specs:
            tickets.append(svc.submit(s, MAX_ITER))
            h2d += mesh_bytes(s)
    keep_t = {tickets[i]: i for i in keep if i < len(tickets)}
    kept = {}
    finished = {}
    remaining = len(specs)
    tick_log = []  # (active cases before the tick, device ms of the tick)
    clock = s0["clock_ms"]
    active = len(specs)
    for _ in range(args.steps):
        for _ in range(args.ticks):
            if remaining == 0:
                break
            nr, nq, _ = svc.step()
            c1 = svc.stats()["clock_ms"]
            tick_log.append((active, c1 - clock))
            clock, active = c1, nr
            d2h += nr * STEP_D2H
            for t in svc.poll():
                st = svc.status(t)
                if e2e:
                    if st["state"] == "converged":
                        u, p = svc.field(t, "U"), svc.field(t, "p")
                        d2h += u.nbytes + p.nbytes
                        if t in keep_t:
                            kept[keep_t[t]] = (u, p)
                    svc.release(t)
                finished[t] = st
                remaining -= 1
    ev1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    ms = ev0.elapsed_time(ev1)
    barrier(ws)
    clocks = clk.stop() if clk else None
    s1 = svc.stats()
    conv = [st for st in finished.values() if st["state"] == "converged"]
    out = dict(ms=ms, wall=wall, converged=len(conv), cases=len(specs), complete=remaining == 0,
               ttc=[st["latency_ms"] for st in conv], iters=[st["iterations"] for st in conv],
               stopped=sum(1 for st in finished.values() if st["state"] != "converged"),
               launches=s1["graph_launches"] - s0["graph_launches"],
               graph_ticks=s1["graph_ticks"] - s0["graph_ticks"], ticks=s1["steps"] - s0["steps"],
               captures=s1["captures"] - s0["captures"], slot_drops=s1["slot_drops"] - s0["slot_drops"],
               host_ms={k: round(s1[k] - s0[k], 1) for k in ("host_rebuild_ms", "host_capture_ms", "host_drop_ms",
                                                            "build_wall_ms", "build_agg_ms", "build_color_ms",
                                                            "build_ell_ms", "build_alloc_ms", "host_admit_ms")},
               peak_bytes=s1["resident_bytes"], h2d=h2d, d2h=d2h, clocks=clocks,
               tickets=tickets, tail=tail_profile(tick_log, len(specs)), admit_s=admit_s,
               cta_rows=s1["cta_rows"], tunes=s1["tunes"], kept=kept,
               first_tick_ms=tick_log[0][1] if tick_log else None)
    return svc, out


def tail_profile(tick_log, cases):
    """How the batch's device time divides between ticks by the number of cases still active:
    the tail of a fixed batch (its last, largest cases alone) is work at low occupancy."""
    tot = sum(ms for _, ms in tick_log) or 1.0
    bands = ((cases // 2, cases + 1), (cases // 8, cases // 2), (16, cases // 8), (0, 16))
    out = []
    for lo, hi in bands:
        sel = [ms for a, ms in tick_log if lo <= a < hi]
        out.append({"active_cases": f"{lo}-{hi - 1}", "ticks": len(sel), "ms": round(sum(sel), 1),
                    "share": round(sum(sel) / tot, 4),
                    "ms_per_tick_median": round(statistics.median(sel), 3) if sel else None})
    return out


ROOF_KERNEL = (1, "k_mc32_l0 (FP32 multicolour Gauss-Seidel sweep of the V-cycle's level 0, "
                  "colour-permuted ELL; one unit = both colours forward then backward over every case)")

# DRAM traffic per byte of the bytes model, from ncu captures of each unit's kernels on a
# 160-case batch (profiles/k_uface_int_bnd_k_assemble_u_cavity_batch.md: k_uface_int + 3 x
# (k_uface_bnd + k_assemble_u) moved 3922.4 MB against 1025.7 MB of the model;
# profiles/k_mc32_level0_cavity_sweep.md: 176.4 MB against 188.3 MB). Traffic grows in
# proportion to the batch, so the live unit's traffic is this ratio times its model bytes.
TRAFFIC_PER_MODEL_BYTE = {3: 3922.4 / 1025.7, 1: 176.4 / 188.3}

# Units of the service's profiling hook: (id, name, units per tick as a function of the tick's U
# smoother sweeps and p V-cycles, bound)
TICK_UNITS = (
    (0, "k_mc64_items (FP64 multicolour Gauss-Seidel sweep of U, ELL copy)", lambda us, pc: us, "hbm"),
    (1, "k_mc32_l0 (FP32 multicolour Gauss-Seidel sweep of the V-cycle's level 0, pre and post)",
     lambda us, pc: 2 * pc, "hbm"),
    (2, "k_fcg_q (FP64 q = A p with (p, q) and (p, r), one per V-cycle)", lambda us, pc: pc, "hbm"),
    (6, "k_coarse_vcycle_pk (the levels below the grid levels, one CTA per large case or 4 small ones)",
     lambda us, pc: pc, "latency"),
    (3, "k_uface_int + k_uface_bnd + k_assemble_u + k_du_boundary (momentum assembly, 3 components)",
     lambda us, pc: 1, "hbm"),
    (4, "k_rhiechow + k_assemble_p (Rhie-Chow face flux and p matrix, 2 correctors)", lambda us, pc: 2, "hbm"),
    (5, "k_bc_update + k_grad_cells + k_grad_bfix + k_minmax_U (field update: gradients of U and p)",
     lambda us, pc: 1, "hbm"),
)


def main_profile(args):
    """ncu target: the kernels of one unit of the roofline kernel and of one eager step."""
    import torch
    from matlab_ufvm_b200 import build as _b
    torch.cuda.set_device(0)
    _b.build()
    settings = service_settings()
    settings.service_eager = 1
    from matlab_ufvm_b200 import ufvm
    svc = ufvm.Service(settings, max_resident_cells=args.budget)
    svc.set_schedule(8192)
    for s in batch_specs(WARM_SEED, args.profile_cases):
        svc.submit(s, MAX_ITER)
    svc.admit()
    nr = 0
    for _ in range(args.warmup * args.ticks):
        nr, nq, _ = svc.step()
        for t in svc.poll():
            svc.release(t)
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


def roofline(svc, peaks, ticks: int = 12):
    """Every major kernel of the tick, timed live on the resident batch with CUDA events (the
    service's profiling hook), with its share of the measured tick; the line's roofline is the
    largest of them. Leaves the batch fit only for timing (the assembly units rewrite fields)."""
    import torch
    stream = torch.cuda.ExternalStream(svc.stream())
    s0 = svc.stats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(ticks):
        svc.step()
    e1.record(stream)
    torch.cuda.synchronize()
    s1 = svc.stats()
    gt = max(1, s1["graph_ticks"] - s0["graph_ticks"])
    tick_ms = e0.elapsed_time(e1) / ticks
    us = (s1["u_loop_bodies"] - s0["u_loop_bodies"]) / gt
    pc = (s1["p_loop_bodies"] - s0["p_loop_bodies"]) / gt
    peak = peaks.get("hbm_gbs")
    rows = []
    for kid, name, per_tick, bound in TICK_UNITS:
        ms, by = svc.profile(kid, 10)
        a = by / (ms * 1e-3) / 1e9
        t = ms * per_tick(us, pc)
        rows.append({"kernel": name, "bound": bound, "ms_per_unit": round(ms, 4), "bytes_per_unit": by,
                     "achieved": round(a, 1), "frac": round(a / peak, 4) if peak else None,
                     "units_per_tick": round(per_tick(us, pc), 2), "ms_per_tick": round(t, 3),
                     "share_of_tick": round(t / tick_ms, 4) if tick_ms > 0 else None})
    top = max(rows, key=lambda r: r["ms_per_tick"])
    top_hbm = max((r for r in rows if r["bound"] == "hbm"), key=lambda r: r["ms_per_tick"])
    top_id = next(kid for kid, name, _, _ in TICK_UNITS if name == top_hbm["kernel"])
    ratio = TRAFFIC_PER_MODEL_BYTE.get(top_id)
    traffic = round(ratio * top_hbm["bytes_per_unit"]) if ratio else None
    return {"kernel": top_hbm["kernel"], "bound": "hbm", "achieved": top_hbm["achieved"], "peak": peak,
            "unit": "GB/s", "frac": top_hbm["frac"], "traffic": traffic,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum on a 160-case batch, scaled to this "
                              "batch by the bytes model" if traffic else None,
            "bytes_per_unit": top_hbm["bytes_per_unit"],
            "ms_per_unit": top_hbm["ms_per_unit"], "share_of_tick": top_hbm["share_of_tick"],
            "largest_kernel_of_tick": top["kernel"],
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if not peaks.get("fallback")
            else "fallback 6650 GB/s (MEASURED_PEAKS.json absent)",
            "tick_ms": round(tick_ms, 3), "u_sweeps_per_tick": round(us, 2), "p_cycles_per_tick": round(pc, 2),
            "kernels": rows}


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


# ------------------------------------------------------------------ the CPU arm (the oracle)
def oracle_fixture(path=ORACLE_FIXTURE):
    """The oracle on a stratified 64-case sample of the batch, converged on the machine that wrote
    the fixture: its own iteration counts and seconds to each residual decade."""
    with open(path) as f:
        d = json.load(f)
    d["sample_cases"] = [c for c in d["cases"] if c["sample"]]
    return d


def _oracle_first3(arg):
    """Seconds of the first three SIMPLE iterations of the oracle (one core) on a batch case."""
    n, re = arg
    from matlab_ufvm_b200 import case
    from oracle import oracle
    spec = case.cavity_case(n, nu=1.0 / re, quirks=case.QUIRKS_CONVERGING, tol_u=0.0, tol_p=0.0)
    oc = oracle.OracleCase(spec)
    t0 = time.perf_counter()
    for _ in range(3):
        oc.iterate()
    return time.perf_counter() - t0


def _oracle_converge(arg):
    """The oracle to convergence (residualControl 1e-6) on one core: (seconds, iterations, state)."""
    n, re = arg
    from matlab_ufvm_b200 import case
    from oracle import oracle
    spec = case.cavity_case(n, nu=1.0 / re, quirks=case.QUIRKS_CONVERGING)
    oc = oracle.OracleCase(spec)
    t0 = time.perf_counter()
    for it in range(1, MAX_ITER + 1):
        rc, _ = oc.iterate()
        if rc != 0:
            return time.perf_counter() - t0, it, "converged" if rc == 1 else "diverged"
    return time.perf_counter() - t0, MAX_ITER, "stopped"


def cpu_batch_estimate(pool, workers: int, fix) -> dict:
    """Converged cases/s of the 512-case batch on `workers` host cores, one case per core.

    Each of the 64 sample cases (every 8th case of the batch ranked by n) contributes its measured
    single-core time to converge, taken from the fixture's full run and carried to this machine by
    the ratio of the first three iterations timed here now (all workers busy, as in the batch) to
    the same iterations on the fixture's machine. A case on which the oracle diverged contributes
    the time it ran until the divergence and no converged case. The batch's total is 512/64 of the
    sample's; the cores are assumed perfectly packed (the longest case alone is far shorter than
    total / cores), which favours the CPU."""
    sample = fix["sample_cases"]
    t3 = pool.map(_oracle_first3, [(c["n"], c["re"]) for c in sample])
    times, conv, ratios = [], 0, []
    for c, t in zip(sample, t3):
        ratio = t / c["seconds_first3"]
        ratios.append(ratio)
        if "diverged_at" in c or "6" not in c.get("seconds_to", {}):
            times.append(c["seconds"] * ratio)
        else:
            times.append(c["seconds_to"]["6"] * ratio)
            conv += 1
    total = sum(times) * SWEEP / len(sample)
    wall = max(total / workers, max(times))
    converged = SWEEP * conv / len(sample)
    return {"cases_per_s": converged / wall, "batch_seconds": wall, "converged_cases": converged,
            "core_seconds": total, "sample_cases": len(sample), "sample_converged": conv,
            "speed_ratio_median": statistics.median(ratios),
            "sample_time_s": sum(t3), "per_case": times}


def cpu_model_check(pool, fix, est: dict, limit_s: float = 3.0) -> dict:
    """Converges the sample cases whose predicted time is under `limit_s` on this machine and
    compares the measured seconds with the prediction of cpu_batch_estimate."""
    pick = [(c, p) for c, p in zip(fix["sample_cases"], est["per_case"])
            if p < limit_s and "diverged_at" not in c and "6" in c.get("first", {})]
    res = pool.map(_oracle_converge, [(c["n"], c["re"]) for c, _ in pick])
    rows = []
    for (c, pred), (sec, it, state) in zip(pick, res):
        rows.append({"n": c["n"], "re": round(c["re"], 1), "iterations": it, "fixture_iterations": c["first"]["6"],
                     "measured_s": round(sec, 4), "predicted_s": round(pred, 4), "state": state})
    ratios = [r["measured_s"] / r["predicted_s"] for r in rows if r["predicted_s"] > 0]
    return {"cases": len(rows), "iterations_match": all(r["iterations"] == r["fixture_iterations"] for r in rows),
            "measured_over_predicted": {"median": statistics.median(ratios) if ratios else None,
                                        "min": min(ratios) if ratios else None,
                                        "max": max(ratios) if ratios else None},
            "measured_total_s": round(sum(r["measured_s"] for r in rows), 3),
            "predicted_total_s": round(sum(r["predicted_s"] for r in rows), 3)}


def cpu_workers(args) -> int:
    return args.cpu_workers or min(os.cpu_count() or 1, 64)


def cpu_sample_text(workers, est) -> str:
    return (f"C++ oracle (serial restatement of the reference's SIMPLE loop with its own V-cycle AMG + "
            f"Gauss-Seidel for p and DILU for U) on {workers} concurrent processes: the first 3 SIMPLE "
            f"iterations of each of the {est['sample_cases']} stratified sample cases of the 512-case batch "
            f"timed here, scaled to each case's fully measured single-core time to convergence "
            f"(tests/golden/sweep_oracle.json; median speed ratio here/there {est['speed_ratio_median']:.3f}); "
            f"{est['sample_converged']}/{est['sample_cases']} sample cases converge in the oracle; "
            f"batch total / cores, perfectly packed")


def pct(v, q):
    return float(np.percentile(np.asarray(v), q)) if len(v) else None


def workload_config(args):
    return {"workload": "512-case batched 2D lid-driven cavity sweep: n log-uniform 16..256 (256-65,536 cells), "
                        "Re uniform 50..1000, seed 2024 (rank r: 2024 + r), SIMPLE to scaled residuals 1e-6, "
                        "every case converged inside the timed region",
            "cases_per_gpu": SWEEP, "ticks_per_step": args.ticks, "resident_cells_per_gpu_cap": args.budget,
            "l2": "inputs larger than L2 (about 5.7M resident cells, GBs of matrices and fields)",
            "parallelism": f"case-sharded x{args.gpus} (one batch per GPU)"}


# ------------------------------------------------------------------ arms
def main_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import multiprocessing as mp
    from oracle import oracle
    oracle.build()
    fix = oracle_fixture()
    workers = cpu_workers(args)
    with mp.get_context("spawn").Pool(workers) as pool:
        check = None
        for w in range(args.warmup):
            est = cpu_batch_estimate(pool, workers, fix)
            if w == 0:
                check = cpu_model_check(pool, fix, est)
        vals = []
        t0 = time.perf_counter()
        for _ in range(args.steps):
            est = cpu_batch_estimate(pool, workers, fix)
            vals.append(est["cases_per_s"])
        el = time.perf_counter() - t0
    v = statistics.median(vals)
    line = {
        "impl": "reference", "metric": "converged_cases_per_s", "value": v, "unit": "cases/s",
        "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args),
        "cpu_baseline": {"value": v, "unit": "cases/s", "cores": workers, "kind": "port",
                         "sample": cpu_sample_text(workers, est)},
        "e2e": {"value": v, "unit": "cases/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "batch_seconds": est["batch_seconds"], "converged_cases": est["converged_cases"],
        "model_check": check,
    }
    print(json.dumps(line), flush=True)
    return 0


def _plain_first3(spec):
    import torch
    from matlab_ufvm_b200 import ufvm
    g = ufvm.GpuCase(spec)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(3):
        g.iterate()
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    g.close()
    return el


def plain_batch_estimate(fix) -> dict:
    """The plain FP64 form one case at a time: the reference's algorithm in FP64 on the GPU (AMG
    rebuilt every p solve, V-cycle with multicolour Gauss-Seidel for p, level-scheduled DILU for U),
    bit-exact with the oracle run with the same settings, so with that run's iteration counts
    (tests/golden/sweep_oracle_plain.json). Each sample case's first three iterations are timed on
    the GPU and scaled by the fixture's measured time to convergence over its first three
    iterations' time; the batch's total is 512/64 of the sample's."""
    from matlab_ufvm_b200 import case
    sample = fix["sample_cases"]
    _plain_first3(case.cavity_case(16, nu=0.01, quirks=case.QUIRKS_CONVERGING, **PLAIN_SETTINGS))  # warm the path
    times, conv, per_iter = [], 0, {}
    for c in sample:
        spec = dataclasses.replace(base_spec(c["n"]), nu=1.0 / c["re"], tol_u=0.0, tol_p=0.0, **PLAIN_SETTINGS)
        t3 = _plain_first3(spec)
        per_iter[str(c["n"])] = round(t3 / 3, 6)
        ratio = t3 / c["seconds_first3"]
        if "diverged_at" in c or "6" not in c.get("seconds_to", {}):
            times.append(c["seconds"] * ratio)
        else:
            times.append(c["seconds_to"]["6"] * ratio)
            conv += 1
    total = sum(times) * SWEEP / len(sample)
    # model check: the smallest sample cases converged on the GPU, measured against the prediction
    check = []
    budget = 20.0
    for c, pred in sorted(zip(sample, times), key=lambda x: x[1]):
        if pred > budget or "diverged_at" in c or "6" not in c.get("first", {}):
            continue
        import torch
        from matlab_ufvm_b200 import ufvm
        spec = dataclasses.replace(base_spec(c["n"]), nu=1.0 / c["re"], **PLAIN_SETTINGS)
        g = ufvm.GpuCase(spec)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        it, _ = g.cfdRunCase(MAX_ITER)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        g.close()
        check.append({"n": c["n"], "re": round(c["re"], 1), "iterations": it, "oracle_iterations": c["first"]["6"],
                      "measured_s": round(el, 4), "predicted_s": round(pred, 4)})
        budget -= el
    ratios = [r["measured_s"] / r["predicted_s"] for r in check if r["predicted_s"] > 0]
    return {"cases_per_s": SWEEP * conv / len(sample) / total, "batch_seconds": total,
            "s_per_iter_first3": per_iter,
            "model_check": {"cases": len(check),
                            "iterations_match_oracle": all(r["iterations"] == r["oracle_iterations"] for r in check),
                            "measured_over_predicted_median": statistics.median(ratios) if ratios else None,
                            "rows": check}}


def plain_kernel_rooflines(peaks, spec=None):
    """The plain FP64 form's solver kernels on the 1,029,000-cell tet channel's momentum matrix
    (device arrays), kernel time only: the library's profiling entry point prepares schedules,
    colourings and the DILU factor, then times each launch with CUDA events after a read of
    twice the L2 size."""
    import torch
    from matlab_ufvm_b200 import case, ufvm
    spec = spec or case.channel_case()
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


def plain_named_configs(channel=None):
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
            ("C2_cavity_64cubed_ilu", lambda: case.cavity_case(64, nu=1.0 / 400, dim=3, p_smoother="ILU"), 2, 1),
            ("C3_channel_1M_tet", lambda: channel or case.channel_case(), 1, 1)):
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


ORACLE_FIELDS = os.path.join(ROOT, "tests", "golden", "sweep_oracle_fields.npz")


def oracle_pinned(rank: int):
    """The pinned cases of the oracle fixture (cases of the seed-2024 batch run by the oracle to
    their fixed point), for the rank whose batch that is."""
    if rank != 0 or not os.path.exists(ORACLE_FIELDS):
        return []
    return [c for c in oracle_fixture()["cases"] if c["pinned"] and "diverged_at" not in c]


def error_vs_oracle(pinned, specs, kept):
    """Relative L2 distance of the bench's converged U and of p - p[cell 0] (read back in the e2e
    pass, at the bench's residualControl stop of 1e-6) from the oracle's fixed point of the same
    case, next to the oracle's own distance at its 1e-6 stop; and, where the fixture holds the
    oracle's 1e-6 fields, the distance between the two 1e-6 stops."""
    import numpy as np
    z = np.load(ORACLE_FIELDS)
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    rows = []
    for c in pinned:
        i = c["index"]
        if i not in kept:
            continue
        nc = specs[i].mesh.n_cells
        U = kept[i][0].reshape(3, -1)[:, :nc]
        p = kept[i][1][:nc]
        Uf, pf = z[f"U_fix_{i}"].astype(np.float64), z[f"p_fix_{i}"].astype(np.float64)
        row = {"index": i, "n": c["n"], "u": rel(U, Uf), "p": rel(p - p[0], pf - pf[0]),
               "u_oracle_own": c["err_u"]["6"], "p_oracle_own": c["err_p"]["6"]}
        if f"U_6_{i}" in z.files:
            U6, p6 = z[f"U_6_{i}"].astype(np.float64), z[f"p_6_{i}"].astype(np.float64)
            row["u_same_rule"] = rel(U, U6)
            row["p_same_rule"] = rel(p - p[0], p6 - p6[0])
        rows.append(row)
    if not rows:
        return None
    q = lambda k: {"p50": pct([r[k] for r in rows], 50), "max": max(r[k] for r in rows)}
    same = [r for r in rows if "u_same_rule" in r]
    out = {"cases": len(rows), "u_rel_l2": q("u"), "p_rel_l2": q("p"),
           "u_over_oracle_own": {"min": min(r["u"] / r["u_oracle_own"] for r in rows),
                                 "max": max(r["u"] / r["u_oracle_own"] for r in rows)},
           "p_over_oracle_own": {"min": min(r["p"] / r["p_oracle_own"] for r in rows),
                                 "max": max(r["p"] / r["p_oracle_own"] for r in rows)},
           "what": "relative L2 of U and of p - p[cell 0] at the bench's 1e-6 stop against the oracle's "
                   "fixed point of the same case (the pinned cases of tests/golden/sweep_oracle.json, "
                   "one per (n, Re) grid point); u/p_over_oracle_own: that error over the oracle's own "
                   "distance from its fixed point at its 1e-6 stop"}
    if same:
        out["same_rule"] = {"cases": len(same), "u_max": max(r["u_same_rule"] for r in same),
                            "p_max": max(r["p_same_rule"] for r in same),
                            "what": "the bench's 1e-6 fields against the oracle's 1e-6 fields (n <= 128)"}
    return out


def main_ours(args):
    import torch
    rank, ws, local = dist_setup(args) if args.gpus > 1 or int(os.environ.get("WORLD_SIZE", "1")) > 1 \
        else (0, 1, 0)
    if not torch.cuda.is_available():
        print(json.dumps({"error": "no CUDA device"}), flush=True)
        return 1
    if ws == 1:
        torch.cuda.set_device(0)
    from matlab_ufvm_b200 import build as _b, sharding
    _b.build()
    seed = sharding.batch_seed(rank, ws, SEED0)
    prebuild_meshes([n for n, _ in batch_params(seed)] + [n for n, _ in batch_params(WARM_SEED)], ws)
    specs = batch_specs(seed)
    peaks = load_peaks()
    wsvc = warm_up(args)
    roof = roofline(wsvc, peaks) if rank == 0 else None
    wsvc.close()
    svc, res = run_batch(args, specs, ws, e2e=False, rank=rank)
    svc.close()
    total = reduce_sum(res["converged"], ws)
    ms = reduce_max(res["ms"], ws)
    value = total / (ms * 1e-3) if ms > 0 else 0.0
    ttc = gather_list(res["ttc"], ws)
    iters = gather_list(res["iters"], ws)
    e2e = None
    pinned = oracle_pinned(rank) if os.path.exists(ORACLE_FIXTURE) else []
    errors = None
    if not args.no_e2e:
        svc2, r2 = run_batch(args, specs, ws, e2e=True, rank=rank, keep=[c["index"] for c in pinned])
        svc2.close()
        if pinned:
            errors = error_vs_oracle(pinned, specs, r2["kept"])
        tot2 = reduce_sum(r2["converged"], ws)
        wall2 = reduce_max(r2["wall"], ws)
        e2e = {"value": tot2 / wall2 if wall2 > 0 else 0.0, "unit": "cases/s",
               "h2d_bytes_per_step": int(reduce_sum(r2["h2d"], ws) / args.steps),
               "d2h_bytes_per_step": int(reduce_sum(r2["d2h"], ws) / args.steps),
               "wall_s": round(r2["wall"], 3), "device_s": round(r2["ms"] * 1e-3, 3),
               "device_s_in_ticks": round(sum(b["ms"] for b in r2["tail"]) * 1e-3, 3),
               "first_tick_ms": r2["first_tick_ms"], "complete": bool(r2["complete"]),
               "ticks_by_active_cases": r2["tail"], "cta_rows": r2["cta_rows"]}
    plain = cpu = check = None
    if rank == 0 and ws == 1:
        fix = oracle_fixture() if os.path.exists(ORACLE_FIXTURE) else None
        if not args.no_cpu and fix:
            import multiprocessing as mp
            from oracle import oracle
            oracle.build()
            workers = cpu_workers(args)
            with mp.get_context("spawn").Pool(workers) as pool:
                cpu = cpu_batch_estimate(pool, workers, fix)
            cpu["workers"] = workers
        if not args.no_plain:
            from matlab_ufvm_b200 import case
            plain = plain_batch_estimate(oracle_fixture(PLAIN_FIXTURE)) if os.path.exists(PLAIN_FIXTURE) else {}
            channel = case.channel_case()
            plain["kernels"] = plain_kernel_rooflines(peaks, channel)
            plain["named"] = plain_named_configs(channel)
    launches = int(reduce_sum(res["launches"], ws))
    if rank == 0:
        line = {
            "metric": "converged_cases_per_s", "value": value, "unit": "cases/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
            "data": "synthetic (seeded cavity meshes generated in-process)",
            "config": workload_config(args),
            "batch_complete": bool(res["complete"]), "converged": int(total), "cases": SWEEP * ws,
            "stopped": int(reduce_sum(res["stopped"], ws)),
            "time_to_converge_ms": {"p50": pct(ttc, 50), "p99": pct(ttc, 99), "n": len(ttc),
                                    "clock": "service device clock, admission to convergence"},
            "iterations": {"p50": pct(iters, 50), "max": max(iters) if iters else None},
            "ticks_timed": res["ticks"], "graph_ticks": res["graph_ticks"], "graph_captures": res["captures"],
            "slot_drops": res["slot_drops"], "resident_bytes_end": res["peak_bytes"],
            "ticks_by_active_cases": res["tail"], "host_ms_in_timed_region": res["host_ms"],
            "device_ms_in_ticks": round(sum(b["ms"] for b in res["tail"]), 1),
            "admission_s_before_timing": round(res["admit_s"], 3) if res["admit_s"] is not None else None,
            "first_tick_ms": res["first_tick_ms"], "cta_rows": res["cta_rows"],
            "roofline": roof, "e2e": e2e, "gpu_launches": launches, "clocks": res["clocks"],
            "error_vs_oracle": errors,
        }
        if cpu:
            line["cpu_baseline"] = {
                "value": cpu["cases_per_s"], "unit": "cases/s", "cores": cpu["workers"], "kind": "port",
                "sample": cpu_sample_text(cpu["workers"], cpu), "batch_seconds": round(cpu["batch_seconds"], 1)}
        if plain:
            line["plain_fp64_gpu"] = {
                "value": plain.get("cases_per_s"), "unit": "cases/s",
                "method": "plain FP64 form one case at a time (the reference's AMG rebuilt every p solve, V-cycle "
                          "with multicolour Gauss-Seidel for p, level-scheduled DILU for U; bit-exact with the oracle "
                          "run with those settings): each of the 64 sample cases' first 3 iterations timed on the "
                          "GPU, scaled by that oracle run's measured time to convergence over its first 3 "
                          "iterations (tests/golden/sweep_oracle_plain.json)",
                "batch_seconds": plain.get("batch_seconds"),
                "s_per_iter_first3": plain.get("s_per_iter_first3"), "model_check": plain.get("model_check"),
                "kernels_1M_tet_channel": plain["kernels"], "named_configs": plain["named"]}
            if plain.get("cases_per_s"):
                line["batched_over_plain"] = value / plain["cases_per_s"]
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

    settings = service_settings()

    def service():
        svc = ufvm.Service(settings, max_resident_cells=args.budget)
        svc.set_admit_interval(args.admit_interval)
        return svc

    svc = service()
    cap = serving.closed_loop_capacity(svc, cap_reqs, args.capacity_steps, spec_fn=spec_fn,
                                       max_iter=args.serving_max_iter)
    cap["stats"] = {k: v for k, v in svc.stats().items() if k in ("resident_bytes", "memory_budget",
                                                                  "deferred_for_memory", "oom_requeues",
                                                                  "footprint_scale", "captures", "slot_drops")}
    svc.close()
    rate = 0.8 * cap["cases_per_s"]
    line = {"workload": "serving mix (70% 2D cavities 1k-64k cells, 25% 3D cavities 32^3-96^3, 5% tet channels "
                        "0.5-2M cells, Re 50..1000, seeded)", "n_gpus": 1, "budget_cells": args.budget,
            "capacity": cap, "arrival_rate_per_s": rate}
    if rate > 0:
        svc = service()
        arr = serving.poisson_arrivals(len(open_reqs), rate, seed=303)
        ol = serving.OpenLoop(svc, open_reqs, arr, spec_fn=spec_fn, max_iter=args.serving_max_iter)
        out = ol.run()
        line["open_loop_stats"] = {k: v for k, v in svc.stats().items() if k in (
            "resident_bytes", "memory_budget", "deferred_for_memory", "oom_requeues", "footprint_scale",
            "captures", "slot_drops", "steps")}
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
