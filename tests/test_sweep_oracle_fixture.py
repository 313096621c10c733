"""The oracle fixtures of the 512-case cavity batch (tests/golden/sweep_oracle.json,
sweep_oracle_fields.npz, sweep_oracle_plain.json): their structure, and one pinned case and
one sample case re-run in the oracle here, which must give the same iteration counts and the
same fixed-point fields (the oracle is deterministic; the stored fields are float32)."""
import json
import os

import numpy as np

from helpers import GOLDEN
from matlab_ufvm_b200 import case


def _load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def test_fixture_structure():
    d = _load("sweep_oracle.json")
    params = case.batched_sweep_params(512, seed=2024)
    sample = [c for c in d["cases"] if c["sample"]]
    assert len(sample) == 64
    pinned = [c for c in d["cases"] if c["pinned"]]
    assert len(pinned) + len(d.get("missing", [])) >= 15
    for c in d["cases"]:
        n, re = params[c["index"]]
        assert (c["n"], round(c["re"], 9)) == (n, round(re, 9))
        assert "diverged_at" not in c  # with QUIRKS_CONVERGING every case of the subset converges
        its = [c["first"][k] for k in sorted(c["first"], key=int)]
        assert its == sorted(its) and its[0] > 0
    z = np.load(os.path.join(GOLDEN, "sweep_oracle_fields.npz"))
    for c in pinned:
        assert z[f"U_fix_{c['index']}"].shape == (3, c["cells"])
    plain = _load("sweep_oracle_plain.json")
    assert sorted(c["index"] for c in plain["cases"]) == sorted(c["index"] for c in sample)


def _rerun(c, tol_k, extra=None):
    from oracle import oracle
    spec = case.cavity_case(c["n"], nu=1.0 / c["re"], quirks=case.QUIRKS_CONVERGING, tol_u=0.0, tol_p=0.0,
                            **(extra or {}))
    oc = oracle.OracleCase(spec)
    first = {}
    for it in range(1, 100000):
        _, res = oc.iterate()
        worst = max(res[:4])
        for k in range(6, tol_k + 1):
            if k not in first and worst <= 10.0 ** -k:
                first[k] = it
        if tol_k in first:
            return first, oc


def test_smallest_pinned_case_reproduces(oracle_mod):
    d = _load("sweep_oracle.json")
    c = min((c for c in d["cases"] if c["pinned"]), key=lambda c: c["first"]["6"] * c["cells"])
    kmax = max(int(k) for k in c["first"])
    first, oc = _rerun(c, kmax)
    assert {str(k): v for k, v in first.items()} == c["first"]
    z = np.load(os.path.join(GOLDEN, "sweep_oracle_fields.npz"))
    nc = c["cells"]
    U = oc.get("U").reshape(3, -1)[:, :nc].astype(np.float32)
    p = oc.get("p")[:nc].astype(np.float32)
    assert np.array_equal(U, z[f"U_fix_{c['index']}"]) and np.array_equal(p, z[f"p_fix_{c['index']}"])


def test_smallest_plain_sample_case_reproduces(oracle_mod):
    d = _load("sweep_oracle_plain.json")
    c = min(d["cases"], key=lambda c: c["first"]["6"] * c["cells"])
    first, _ = _rerun(c, 6, {"p_smoother": "MCGS"})
    assert first[6] == c["first"]["6"]


def test_bench_error_vs_oracle_reads_the_fixture():
    """bench.py's error_vs_oracle on fields whose distances are known: the oracle's own 1e-6
    fields (where the fixture holds them) are as far from the fixed point as the fixture says,
    and at distance zero from themselves under the same rule."""
    import importlib.util
    import types
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("ufvm_bench", os.path.join(root, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    z = np.load(os.path.join(GOLDEN, "sweep_oracle_fields.npz"))
    pinned = [c for c in bench.oracle_pinned(0) if f"U_6_{c['index']}" in z.files]
    assert len(pinned) >= 8
    specs = {c["index"]: types.SimpleNamespace(mesh=types.SimpleNamespace(n_cells=c["cells"])) for c in pinned}
    kept = {c["index"]: (z[f"U_6_{c['index']}"].astype(np.float64).reshape(-1),
                         z[f"p_6_{c['index']}"].astype(np.float64)) for c in pinned}
    out = bench.error_vs_oracle(pinned, specs, kept)
    assert out["cases"] == len(pinned) and out["same_rule"]["u_max"] == 0.0 and out["same_rule"]["p_max"] == 0.0
    # the stored 1e-6 fields are float32: their distance matches the fixture's FP64 one to rounding
    assert 0.999 < out["u_over_oracle_own"]["min"] <= out["u_over_oracle_own"]["max"] < 1.001
    assert 0.99 < out["p_over_oracle_own"]["min"] <= out["p_over_oracle_own"]["max"] < 1.01
