"""Open-loop serving of steady-case requests: the mixed request stream, Poisson arrivals, and
a driver that feeds a batched service at the arrival times and measures time to converge.

The request mix: 70% 2D lid-driven cavities of 1k-64k cells, 25% 3D cavities of 32^3-96^3
cells, 5% jittered-tet channels of 0.5-2M cells, Re uniform in 50..1000, all seeded. Arrival
times are a Poisson process of a given rate on the service's clock (the accumulated device
time of its steps); when the service has nothing to do, the driver's clock jumps to the next
arrival. A request's time to converge is measured from its arrival:
(submission - arrival) + queue time + admission-to-convergence time, all on that clock.

The driver only uses the service's public calls (submit, step, poll, status, release,
stats), so it runs on ufvm.Service and, in the tests, on a stand-in with the same calls.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

KINDS = ("cavity2d", "cavity3d", "channel")
MIX = (0.70, 0.25, 0.05)
CHANNEL_BASE = (140, 35, 35)  # 1,029,000 tets at 6 tets per hex


@dataclasses.dataclass(frozen=True)
class Request:
    index: int
    kind: str
    size: tuple      # (n,) 2D, (m,) 3D, (nx, ny, nz) channel
    re: float

    @property
    def cells(self) -> int:
        if self.kind == "cavity2d":
            return self.size[0] ** 2
        if self.kind == "cavity3d":
            return self.size[0] ** 3
        nx, ny, nz = self.size
        return 6 * nx * ny * nz


def serving_mix(count: int, seed: int = 7, mix: Sequence[float] = MIX, re_range=(50.0, 1000.0),
                cells_2d=(1_000, 64_000), edge_3d=(32, 96), cells_channel=(500_000, 2_000_000)) -> List[Request]:
    """Seeded request stream: kind by `mix`, sizes log-uniform in cells (2D, channel) or in
    edge length (3D), Re uniform."""
    rng = np.random.default_rng(seed)
    cum = np.cumsum(np.asarray(mix, dtype=np.float64))
    cum /= cum[-1]
    out = []
    for i in range(count):
        kind = KINDS[int(np.searchsorted(cum, rng.random(), side="right"))]
        if kind == "cavity2d":
            cells = math.exp(rng.uniform(math.log(cells_2d[0]), math.log(cells_2d[1])))
            size = (int(np.clip(round(math.sqrt(cells)), math.ceil(math.sqrt(cells_2d[0])),
                                math.floor(math.sqrt(cells_2d[1])))),)
        elif kind == "cavity3d":
            size = (int(round(math.exp(rng.uniform(math.log(edge_3d[0]), math.log(edge_3d[1]))))),)
        else:
            cells = math.exp(rng.uniform(math.log(cells_channel[0]), math.log(cells_channel[1])))
            s = (cells / (6.0 * np.prod(CHANNEL_BASE))) ** (1.0 / 3.0)
            size = tuple(max(2, int(round(b * s))) for b in CHANNEL_BASE)
        out.append(Request(i, kind, size, float(rng.uniform(*re_range))))
    return out


def poisson_arrivals(count: int, rate_per_s: float, seed: int = 11) -> np.ndarray:
    """Arrival times (s) of a Poisson process of the given rate, starting at 0."""
    if rate_per_s <= 0:
        raise ValueError("arrival rate must be positive")
    gaps = np.random.default_rng(seed).exponential(1.0 / rate_per_s, size=count)
    return np.concatenate([[0.0], np.cumsum(gaps[:-1])]) if count else np.zeros(0)


def request_spec(req: Request, quirks: Optional[int] = None):
    """The steady case of a request (the same builders as the named workloads)."""
    from matlab_ufvm_b200 import case
    q = case.QUIRKS_CONVERGING if quirks is None else quirks
    nu = 1.0 / req.re
    if req.kind == "cavity2d":
        return case.cavity_case(req.size[0], nu=nu, quirks=q)
    if req.kind == "cavity3d":
        return case.cavity_case(req.size[0], nu=nu, dim=3, quirks=q)
    nx, ny, nz = req.size
    return case.channel_case(nx, ny, nz, nu=nu, quirks=q)


@dataclasses.dataclass
class Outcome:
    index: int
    kind: str
    state: str
    iterations: int
    arrival_s: float
    late_s: float        # submission - arrival (at most one service step)
    queue_s: float
    service_s: float     # admission to convergence (or to the stop)
    size: tuple = ()
    re: float = 0.0
    status: int = 0      # ufvm_status of a stopped request
    residuals: tuple = ()  # rms U1 U2 U3 p at the end

    @property
    def time_to_converge_s(self) -> float:
        return self.late_s + self.queue_s + self.service_s


class OpenLoop:
    """Feeds `svc` with `requests` at `arrival_s` (service clock) and records each outcome."""

    def __init__(self, svc, requests: Sequence[Request], arrival_s: Sequence[float],
                 spec_fn: Callable = request_spec, max_iter: int = 20000, release: bool = True):
        if len(requests) != len(arrival_s):
            raise ValueError("one arrival time per request")
        order = np.argsort(np.asarray(arrival_s, dtype=np.float64), kind="stable")
        self.svc = svc
        self.requests = [requests[i] for i in order]
        self.arrival = [float(arrival_s[i]) for i in order]
        self.spec_fn, self.max_iter, self.release = spec_fn, max_iter, release
        self.idle_s = 0.0         # clock jumps while the service had nothing to do
        self.next = 0
        self.live: Dict[int, tuple] = {}  # ticket -> (request, arrival, submit clock)
        self.idle_at: Dict[int, float] = {}  # ticket -> idle offset of the clock at its submission
        self.outcomes: List[Outcome] = []
        self.steps = 0

    def clock_s(self) -> float:
        return self.svc.stats()["clock_ms"] * 1e-3 + self.idle_s

    def _submit_due(self):
        now = self.clock_s()
        while self.next < len(self.requests) and self.arrival[self.next] <= now:
            req, arr = self.requests[self.next], self.arrival[self.next]
            t = self.svc.submit(self.spec_fn(req), self.max_iter)
            self.live[t] = (req, arr, now)
            self.idle_at[t] = self.idle_s
            self.next += 1

    def _collect(self):
        for t in self.svc.poll():
            if t not in self.live:
                continue
            req, arr, sub = self.live.pop(t)
            st = self.svc.status(t)
            self.outcomes.append(Outcome(req.index, req.kind, st["state"], int(st["iterations"]), arr,
                                         max(0.0, sub - arr), st["queue_ms"] * 1e-3, st["latency_ms"] * 1e-3,
                                         tuple(req.size), float(req.re), int(st.get("status", 0)),
                                         tuple(float(x) for x in list(st.get("res", ()))[:4])))
            if self.release:
                self.svc.release(t)

    def run(self, max_steps: int = 10 ** 9) -> List[Outcome]:
        """Until every request has finished (or max_steps service steps)."""
        while (self.next < len(self.requests) or self.live) and self.steps < max_steps:
            self._submit_due()
            if not self.live:
                # nothing resident or queued: the clock moves on to the next arrival
                self.idle_s += max(0.0, self.arrival[self.next] - self.clock_s())
                continue
            self.svc.step()
            self.steps += 1
            self._collect()
        return self.outcomes


def closed_loop_capacity(svc, requests: Sequence[Request], steps: int, spec_fn: Callable = request_spec,
                         max_iter: int = 20000, depth: int = 64) -> Dict:
    """Converged cases per second of service clock with the queue kept `depth` deep."""
    it = iter(requests)
    live = set()
    queued = 0

    def top_up():
        nonlocal queued
        while queued < depth:
            req = next(it, None)
            if req is None:
                return
            live.add(svc.submit(spec_fn(req), max_iter))
            queued += 1

    top_up()
    t0 = svc.stats()["clock_ms"]
    done = 0
    for _ in range(steps):
        _, nq, _ = svc.step()
        queued = nq
        for t in svc.poll():
            if t in live:
                live.discard(t)
                done += svc.status(t)["state"] == "converged"
                svc.release(t)
        top_up()
    dt = (svc.stats()["clock_ms"] - t0) * 1e-3
    return {"converged": done, "seconds": dt, "cases_per_s": done / dt if dt > 0 else 0.0}


def summarize(outcomes: Sequence[Outcome]) -> Dict:
    """Throughput (converged requests over the span from the first arrival to the last
    convergence) and time-to-converge percentiles, overall and per request kind."""
    def pcts(xs):
        a = np.asarray(xs, dtype=np.float64)
        return {"p50": float(np.percentile(a, 50)) if len(a) else None,
                "p99": float(np.percentile(a, 99)) if len(a) else None, "n": int(len(a))}

    conv = [o for o in outcomes if o.state == "converged"]
    span = (max(o.arrival_s + o.time_to_converge_s for o in conv) - min(o.arrival_s for o in outcomes)) \
        if conv else 0.0
    stopped = [{"index": o.index, "kind": o.kind, "size": list(o.size), "re": round(o.re, 1),
                "iterations": o.iterations, "status": o.status, "rms_residuals": list(o.residuals)}
               for o in outcomes if o.state != "converged"]
    return {"requests": len(outcomes), "converged": len(conv), "stopped": stopped,
            "cases_per_s": len(conv) / span if span > 0 else 0.0,
            "time_to_converge_s": pcts([o.time_to_converge_s for o in conv]),
            "queue_s": pcts([o.late_s + o.queue_s for o in conv]),
            "by_kind": {k: pcts([o.time_to_converge_s for o in conv if o.kind == k]) for k in KINDS}}
