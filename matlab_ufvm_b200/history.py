"""Residual histories of a steady SIMPLE run in the reference's columns.

uFVM keeps the rms residual of each equation component per iteration
(fvm/extras/cfdStoreResiduals.m:13-22) and prints, per component, the rms and max scaled
residuals and the linear solver's residual before and after the solve
(fvm/print/cfdPrintResiduals.m:5-48). A history row here holds the same four numbers for U-x,
U-y, U-z and p, taken from the 16 residuals one SIMPLE iteration returns (ufvm_simple_iteration:
rms U1 U2 U3 p, max (4), linear-solver initial (4), final (4)).
"""
from __future__ import annotations

import json
from typing import Callable, Iterable, List, Sequence, Tuple

COMPONENTS = ("U-x", "U-y", "U-z", "p")
COLUMNS = ("rms", "max", "initial", "final")


def row(iteration: int, res16: Sequence[float]) -> dict:
    """One iteration: for each component, [rms, max, linear-solver initial, final]."""
    r = [float(x) for x in res16]
    return {"iteration": int(iteration),
            **{c: [r[k], r[4 + k], r[8 + k], r[12 + k]] for k, c in enumerate(COMPONENTS)}}


def record(step: Callable[[], Tuple[Sequence[float], bool]], max_iterations: int,
           until_converged: bool = True) -> List[dict]:
    """Runs `step` (one SIMPLE iteration returning (res16, converged)) up to max_iterations times,
    stopping after the iteration that converges when until_converged."""
    out = []
    for it in range(1, max_iterations + 1):
        res, conv = step()
        out.append(row(it, res))
        if until_converged and conv:
            break
    return out


def write_jsonl(path: str, rows: Iterable[dict], meta: dict | None = None) -> None:
    with open(path, "w") as f:
        if meta:
            f.write(json.dumps({"meta": meta}) + "\n")
        for r in rows:
            f.write(json.dumps(r) + "\n")


def side_by_side(a: Sequence[dict], b: Sequence[dict], names=("GPU", "oracle"), every: int = 1) -> str:
    """A Markdown table of two histories, one line per iteration and component (every `every`-th
    iteration and the last), in the reference's print columns."""
    head = (f"| iteration | component | rms {names[0]} | rms {names[1]} | max {names[0]} | max {names[1]} | "
            f"initial {names[0]} | initial {names[1]} | final {names[0]} | final {names[1]} |")
    lines = [head, "|" + "---|" * 10]
    n = min(len(a), len(b))
    for i in range(n):
        if (i + 1) % every and i != n - 1:
            continue
        for c in COMPONENTS:
            x, y = a[i][c], b[i][c]
            cells = [f"{x[k]:.6e} | {y[k]:.6e}" for k in range(4)]
            lines.append(f"| {a[i]['iteration']} | {c} | " + " | ".join(cells) + " |")
    return "\n".join(lines)
