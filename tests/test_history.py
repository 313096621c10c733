"""Residual-history rows in the reference's columns (host logic, no GPU)."""
import json

import numpy as np

from matlab_ufvm_b200 import history


def test_row_layout_follows_the_sixteen_residuals():
    res = np.arange(16, dtype=float)
    r = history.row(3, res)
    assert r["iteration"] == 3
    assert r["U-x"] == [0, 4, 8, 12] and r["U-z"] == [2, 6, 10, 14] and r["p"] == [3, 7, 11, 15]


def test_record_stops_after_convergence_and_writes_jsonl(tmp_path):
    state = {"k": 0}

    def step():
        state["k"] += 1
        return np.full(16, 10.0 ** -state["k"]), state["k"] == 4

    rows = history.record(step, 10, True)
    assert [r["iteration"] for r in rows] == [1, 2, 3, 4]
    assert len(history.record(lambda: (np.zeros(16), True), 3, False)) == 3
    p = tmp_path / "h.jsonl"
    history.write_jsonl(str(p), rows, {"config": "x"})
    lines = p.read_text().splitlines()
    assert json.loads(lines[0]) == {"meta": {"config": "x"}} and json.loads(lines[4])["iteration"] == 4
    table = history.side_by_side(rows, rows, every=2)
    assert table.count("| 2 | U-x |") == 1 and table.count("| 4 | p |") == 1 and "| 1 |" not in table
