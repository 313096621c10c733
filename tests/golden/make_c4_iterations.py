"""Writes c4_sweep_iterations.json: iterations to converge of the 512-case 2D cavity sweep
(batched_sweep_params(512, seed=2024), QUIRKS_CONVERGING, scaled residuals <= 1e-6) in the
batched service. Needs a CUDA GPU; run from the repository root:

    python tests/golden/make_c4_iterations.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from matlab_ufvm_b200 import case, ufvm  # noqa: E402


def main():
    params = case.batched_sweep_params(512)
    specs = [case.cavity_case(n, nu=1.0 / re, quirks=case.QUIRKS_CONVERGING) for (n, re) in params]
    svc = ufvm.Service(ufvm.fast_settings(specs[0]), max_resident_cells=8_000_000)
    tickets = [svc.submit(s, 20000) for s in specs]
    svc.run()
    cases = []
    for (n, re), t in zip(params, tickets):
        st = svc.status(t)
        assert st["state"] == "converged", (n, re, st)
        cases.append({"n": n, "re": round(re, 6), "iterations": st["iterations"]})
    out = {"description": "Iterations to converge (scaled residuals <= 1e-6) of the 512-case 2D cavity sweep "
                          "(batched_sweep_params(512, seed=2024), QUIRKS_CONVERGING) in the batched service: "
                          "FP64 multicolour Gauss-Seidel for U, FP32 AMG preconditioning for p. Written by "
                          "make_c4_iterations.py on a B200.",
           "cases": cases}
    with open(os.path.join(HERE, "c4_sweep_iterations.json"), "w") as f:
        json.dump(out, f, indent=0)


if __name__ == "__main__":
    main()
