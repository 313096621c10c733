"""Residual histories of the plain FP64 form beside the oracle's, row by row, in the reference's
columns (fvm/extras/cfdStoreResiduals.m:13-22, fvm/print/cfdPrintResiduals.m:5-48): rms and max
scaled residuals and the linear solver's initial and final residuals of U-x, U-y, U-z and p.

C1 (20 x 20 cavity, Re 100) runs to convergence (58 iterations); C2 (64^3 cavity, Re 400, ILU
for p) over its first 10 iterations and C3 (1,029,000-cell jittered-tet channel, Re 200) over its
first 4 (windows sized to keep the oracle's single-core time to about a minute each). The
GPU's and the oracle's rows agree to a relative 1e-10 (the rms and max reductions sum in a
different order; everything else is bit-exact). With UFVM_HISTORY_DIR set, both histories are
written there as JSONL and as a side-by-side Markdown table."""
import os

import numpy as np
import pytest

from matlab_ufvm_b200 import case, history

pytestmark = pytest.mark.gpu

RTOL = 1e-10
CONFIGS = {
    "C1_cavity_20x20": (lambda: case.cavity_case(20, nu=0.01), 500, True),
    "C2_cavity_64cubed_ilu": (lambda: case.cavity_case(64, nu=1.0 / 400, dim=3, p_smoother="ILU"), 10, False),
    "C3_channel_1M_tet": (lambda: case.channel_case(), 4, False),
}


@pytest.mark.parametrize("name", list(CONFIGS))
def test_residual_history_side_by_side(ufvm_mod, oracle_mod, name):
    make, iters, to_convergence = CONFIGS[name]
    spec = make()
    g = ufvm_mod.GpuCase(spec)
    hg = history.record(g.iterate, iters, to_convergence)
    g.close()
    oc = oracle_mod.OracleCase(spec)

    def oracle_step():
        rc, res = oc.iterate()
        return res, rc == 1

    ho = history.record(oracle_step, iters, to_convergence)
    assert len(hg) == len(ho)
    if to_convergence:
        assert len(hg) == 58  # C1 converges in the oracle's 58 iterations
    for a, b in zip(hg, ho):
        for c in history.COMPONENTS:
            assert np.allclose(a[c], b[c], rtol=RTOL, atol=0), (name, a["iteration"], c, a[c], b[c])
    out = os.environ.get("UFVM_HISTORY_DIR")
    if out:
        os.makedirs(out, exist_ok=True)
        meta = {"config": name, "cells": spec.mesh.n_cells, "iterations": len(hg)}
        history.write_jsonl(os.path.join(out, f"{name}_gpu.jsonl"), hg, meta)
        history.write_jsonl(os.path.join(out, f"{name}_oracle.jsonl"), ho, meta)
        with open(os.path.join(out, f"{name}.md"), "w") as f:
            f.write(history.side_by_side(hg, ho, every=5 if to_convergence else 1) + "\n")
