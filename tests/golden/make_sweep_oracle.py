"""Writes sweep_oracle.json and sweep_oracle_fields.npz: the FP64 oracle on a seeded subset of
the 512-case 2D cavity sweep (batched_sweep_params(512, seed=2024), QUIRKS_CONVERGING).

The oracle is the single-thread C++ restatement of the reference's steady SIMPLE loop
(top/cfdRunCase.m:92-142) with its own solvers: the V-cycle agglomeration AMG of
solve/AMG/cfdApplyAMG.m with symmetric Gauss-Seidel (solve/cfdSolveSOR.m) for p and DILU
(solve/cfdSolveILU.m) for U. Each case is iterated past the reference's residualControl test
(booleans/cfdCheckConvergence.m:3-20: the rms residuals of U1, U2, U3 and p all <= tol) down to
its fixed point, and the file records, for tol = 1e-6 ... 1e-11, the iteration at which the
test first passes and the distance of the fields at that iteration from the fixed point (the
sample cases that are not pinned only to the tol = 1e-6 stop).

Two subsets of the sweep:

* ``sample``: 64 cases, every 8th case of the sweep ranked by (n, Re) -- a stratified sample of
  the workload's cost distribution. The bench's CPU arm times oracle iterations on these cases
  and multiplies by the oracle's own iteration counts recorded here.
* ``pinned``: for each grid point n in {16, 32, 64, 128, 256} x Re in {50, 500, 1000}, the sweep
  case nearest to it. Their fixed-point fields (U, p over the cells, float32) and, for n <= 128,
  the fields at the tol = 1e-6 stop are stored in the npz: the parity target of the batched
  service at its operating point.

A case on which the oracle diverges (a NaN residual: the reference's divergence test,
top/cfdRunCase.m:124-127) is recorded with the iteration it diverged at and no fields.

With --variant plain the same sample is run with the settings of the plain FP64 GPU form
(multicolour Gauss-Seidel as the AMG smoother for p, the GPU path's UFVM_SMOOTHER_MCGS, whose
restatement in the oracle is bit-exact with it; DILU for U as before), only to the tol = 1e-6
stop, into sweep_oracle_plain.json: the iteration counts and times of the plain form's algorithm.

Long-running (about two hours on 8 cores); per-case results are kept in --parts so an
interrupted run resumes. Run from the repository root:

    python tests/golden/make_sweep_oracle.py [--workers 7] [--parts DIR] [--variant plain]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

DECADES = (6, 7, 8, 9, 10, 11)
GRID_N = (16, 32, 64, 128, 256)
GRID_RE = (50.0, 500.0, 1000.0)
FIELD_SNAPSHOT_MAX_N = 128


def sweep():
    from matlab_ufvm_b200 import case
    return case.batched_sweep_params(512, seed=2024)


def sample_indices(params):
    order = sorted(range(len(params)), key=lambda i: (params[i][0], params[i][1]))
    return sorted(order[k] for k in range(4, len(order), 8))


def pinned_indices(params):
    out = []
    for ng in GRID_N:
        for rg in GRID_RE:
            best = min((i for i in range(len(params)) if i not in out),
                       key=lambda i: (math.log2(params[i][0] / ng)) ** 2 + ((params[i][1] - rg) / 200.0) ** 2)
            out.append(best)
    return out


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def run_case(job):
    idx, n, re, keep_fields, parts, variant = job
    path = os.path.join(parts, f"case{idx:03d}.npz")
    if os.path.exists(path):
        return idx
    from matlab_ufvm_b200 import case
    from oracle import oracle
    extra = {"p_smoother": "MCGS"} if variant == "plain" else {}
    # only the pinned cases are iterated to their fixed point; the sample needs the 1e-6 stop
    decades = DECADES if keep_fields else (6,)
    spec = case.cavity_case(n, nu=1.0 / re, quirks=case.QUIRKS_CONVERGING, tol_u=0.0, tol_p=0.0, **extra)
    oc = oracle.OracleCase(spec)
    nc = spec.mesh.n_cells
    snaps, first, t_first = {}, {}, {}
    best, best_it, it = math.inf, 0, 0
    t3 = None
    t0 = time.perf_counter()
    while True:
        it += 1
        rc, res = oc.iterate()
        if it == 3:
            t3 = time.perf_counter() - t0
        if rc < 0 or not np.all(np.isfinite(res[:4])):
            # the reference's divergence test (top/cfdRunCase.m:124-127): recorded, not raised
            meta = {"index": idx, "n": n, "re": re, "cells": nc, "iterations_run": it,
                    "seconds": time.perf_counter() - t0, "diverged_at": it, "seconds_first3": t3,
                    "first": {str(k): v for k, v in first.items()}}
            tmp = path + ".tmp.npz"
            np.savez(tmp, meta=np.array(json.dumps(meta)))
            os.replace(tmp, path)
            return idx
        worst = float(max(res[0], res[1], res[2], res[3]))
        for k in decades:
            if k not in first and worst <= 10.0 ** -k:
                first[k] = it
                t_first[k] = time.perf_counter() - t0
                snaps[k] = (oc.get("U").reshape(3, -1)[:, :nc].copy(), oc.get("p")[:nc].copy())
        if worst < 0.9 * best:
            best, best_it = worst, it
        i6 = first.get(6)
        if len(first) == len(decades):
            break
        if i6 is not None and (it - best_it > 400 or it > 4 * i6 + 2000):
            break  # stagnated at the floating-point floor
        if it - best_it > 1500 or it > 60000:
            break  # no progress: recorded without the decades it did not reach
    wall = time.perf_counter() - t0
    U = oc.get("U").reshape(3, -1)[:, :nc].copy()
    p = oc.get("p")[:nc].copy()
    pf = p - p[0]
    err_u = {k: rel(s[0], U) for k, s in snaps.items()}
    err_p = {k: rel(s[1] - s[1][0], pf) for k, s in snaps.items()}
    arrays = dict(meta=np.array(json.dumps({
        "index": idx, "n": n, "re": re, "cells": nc, "iterations_run": it, "seconds": wall,
        "final_worst_residual": worst, "first": {str(k): v for k, v in first.items()},
        "seconds_first3": t3, "seconds_to": {str(k): v for k, v in t_first.items()},
        "err_u": {str(k): v for k, v in err_u.items()}, "err_p": {str(k): v for k, v in err_p.items()}})))
    if keep_fields:
        arrays["U_fix"] = U.astype(np.float32)
        arrays["p_fix"] = p.astype(np.float32)
        if n <= FIELD_SNAPSHOT_MAX_N and 6 in snaps:
            arrays["U_6"] = snaps[6][0].astype(np.float32)
            arrays["p_6"] = snaps[6][1].astype(np.float32)
    tmp = path + ".tmp.npz"
    np.savez(tmp, **arrays)
    os.replace(tmp, path)
    return idx


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workers", type=int, default=max(1, (os.cpu_count() or 2) - 1))
    ap.add_argument("--parts", default=os.path.join(tempfile.gettempdir(), "ufvm_sweep_oracle_parts"))
    ap.add_argument("--variant", choices=("reference", "plain"), default="reference")
    ap.add_argument("--assemble-only", action="store_true",
                    help="write the fixture from the per-case results present in --parts, listing any missing case")
    args = ap.parse_args()
    os.makedirs(args.parts, exist_ok=True)
    params = sweep()
    sample, pinned = sample_indices(params), pinned_indices(params)
    if args.variant == "plain":
        pinned = []
    todo = sorted(set(sample) | set(pinned), key=lambda i: -(params[i][0] ** 3))
    jobs = [(i, params[i][0], params[i][1], i in pinned, args.parts, args.variant) for i in todo]
    if not args.assemble_only:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(args.workers) as pool:
            for k, idx in enumerate(pool.imap_unordered(run_case, jobs)):
                print(f"[{k + 1}/{len(jobs)}] case {idx} done", flush=True)
    cases, fields, missing = [], {}, []
    for i in sorted(set(sample) | set(pinned)):
        path = os.path.join(args.parts, f"case{i:03d}.npz")
        if not os.path.exists(path):
            missing.append(i)
            continue
        z = np.load(path)
        meta = json.loads(str(z["meta"]))
        meta["sample"], meta["pinned"] = i in sample, i in pinned
        cases.append(meta)
        for key in ("U_fix", "p_fix", "U_6", "p_6"):
            if key in z.files:
                fields[f"{key}_{i}"] = z[key]
    out = {"description": "FP64 oracle (C++ restatement of the reference's steady SIMPLE loop, V-cycle AMG with "
                          "symmetric Gauss-Seidel for p, DILU for U) on a subset of the 512-case 2D cavity sweep "
                          "batched_sweep_params(512, seed=2024), QUIRKS_CONVERGING. first[k]: iteration at which "
                          "the rms residuals of U1, U2, U3 and p are all <= 10^-k; err_u/err_p[k]: relative L2 "
                          "distance of U / (p - p[0]) at that iteration from the fixed point (the last "
                          "iteration run); seconds: single-thread wall time of the whole run on the generating "
                          "machine, seconds_first3 of its first three iterations, seconds_to[k] up to first[k]; "
                          "diverged_at: the iteration whose residual was NaN. Written by make_sweep_oracle.py.",
           "sample": sample, "pinned": pinned, "grid_n": list(GRID_N), "grid_re": list(GRID_RE),
           "missing": missing, "cases": cases}
    if args.variant == "plain":
        out["description"] = ("The oracle with the plain FP64 GPU form's settings (multicolour Gauss-Seidel as the "
                              "AMG smoother for p, DILU for U) on the 64-case sample of the 512-case 2D cavity sweep, "
                              "to the tol = 1e-6 stop; fields as in sweep_oracle.json. Written by "
                              "make_sweep_oracle.py --variant plain.")
        with open(os.path.join(HERE, "sweep_oracle_plain.json"), "w") as f:
            json.dump(out, f, indent=0)
        return
    with open(os.path.join(HERE, "sweep_oracle.json"), "w") as f:
        json.dump(out, f, indent=0)
    np.savez_compressed(os.path.join(HERE, "sweep_oracle_fields.npz"), **fields)


if __name__ == "__main__":
    main()
