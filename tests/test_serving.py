"""Host logic of the open-loop serving driver, on a stand-in service with the public calls of
ufvm.Service (submit / step / poll / status / release / stats) and a simulated device clock."""
import numpy as np
import pytest

from matlab_ufvm_b200 import serving


class FakeService:
    """FIFO admission by resident cells; each step advances the clock by a time proportional to
    the resident cells; a request converges after a size-dependent number of steps."""

    STEP_MS_PER_MCELL = 40.0

    def __init__(self, budget_cells=4_000_000):
        self.budget = budget_cells
        self.clock = 0.0
        self.queue, self.resident, self.finished = [], {}, []
        self.rec = {}
        self.next_ticket = 1

    @staticmethod
    def steps_needed(req):
        return 3 + req.cells // 200_000

    def submit(self, req, max_iter):
        t = self.next_ticket
        self.next_ticket += 1
        self.rec[t] = dict(req=req, state="queued", it=0, t_submit=self.clock, t_admit=None, t_done=None)
        self.queue.append(t)
        return t

    def step(self):
        cells = sum(self.rec[t]["req"].cells for t in self.resident)
        while self.queue and (cells == 0 or cells + self.rec[self.queue[0]]["req"].cells <= self.budget):
            t = self.queue.pop(0)
            r = self.rec[t]
            r["state"], r["t_admit"] = "resident", self.clock
            self.resident[t] = self.steps_needed(r["req"])
            cells += r["req"].cells
        self.clock += 1.0 + self.STEP_MS_PER_MCELL * cells * 1e-6
        for t in list(self.resident):
            self.rec[t]["it"] += 1
            self.resident[t] -= 1
            if self.resident[t] == 0:
                del self.resident[t]
                self.rec[t].update(state="converged", t_done=self.clock)
                self.finished.append(t)
        return len(self.resident), len(self.queue), len(self.finished)

    def poll(self):
        out, self.finished = self.finished, []
        return out

    def status(self, t):
        r = self.rec[t]
        lat = r["t_done"] - r["t_admit"] if r["t_done"] is not None else 0.0
        q = (r["t_admit"] if r["t_admit"] is not None else self.clock) - r["t_submit"]
        return dict(state=r["state"], iterations=r["it"], latency_ms=lat, queue_ms=q)

    def release(self, t):
        self.rec[t]["released"] = True

    def stats(self):
        return {"clock_ms": self.clock}


def identity(req):
    return req


def test_mix_is_seeded_and_has_the_stated_shares():
    a = serving.serving_mix(3000, seed=3)
    assert a == serving.serving_mix(3000, seed=3) and a != serving.serving_mix(3000, seed=4)
    share = {k: sum(r.kind == k for r in a) / len(a) for k in serving.KINDS}
    assert abs(share["cavity2d"] - 0.70) < 0.03 and abs(share["cavity3d"] - 0.25) < 0.03
    assert abs(share["channel"] - 0.05) < 0.015
    for r in a:
        assert 50 <= r.re <= 1000
        if r.kind == "cavity2d":
            assert 32 <= r.size[0] <= 252 and 1000 <= r.cells <= 64_000
        elif r.kind == "cavity3d":
            assert 32 <= r.size[0] <= 96
        else:
            assert 0.45e6 <= r.cells <= 2.1e6


def test_poisson_arrivals():
    t = serving.poisson_arrivals(20000, rate_per_s=4.0, seed=1)
    assert t[0] == 0.0 and np.all(np.diff(t) >= 0)
    assert abs(np.mean(np.diff(t)) - 0.25) < 0.25 * 0.03
    with pytest.raises(ValueError):
        serving.poisson_arrivals(3, 0.0)


def test_open_loop_accounts_time_from_arrival():
    reqs = serving.serving_mix(120, seed=5)
    arr = serving.poisson_arrivals(len(reqs), rate_per_s=30.0, seed=2)
    svc = FakeService()
    ol = serving.OpenLoop(svc, reqs, arr, spec_fn=identity)
    out = ol.run()
    assert len(out) == len(reqs) and {o.index for o in out} == set(range(len(reqs)))
    by_index = {o.index: o for o in out}
    for t, r in svc.rec.items():
        o = by_index[r["req"].index]
        assert o.state == "converged" and r.get("released")
        assert o.late_s >= 0.0
        # submission - arrival + queue + service = convergence - arrival, on the driver's clock
        assert o.time_to_converge_s == pytest.approx(r["t_done"] * 1e-3 + ol.idle_at[t] - o.arrival_s, abs=1e-9)
    s = serving.summarize(out)
    assert s["converged"] == len(reqs) and s["cases_per_s"] > 0
    assert s["time_to_converge_s"]["p50"] <= s["time_to_converge_s"]["p99"]
    assert sum(v["n"] for v in s["by_kind"].values()) == len(reqs)


def test_open_loop_idles_to_the_next_arrival():
    reqs = serving.serving_mix(10, seed=8, mix=(1.0, 0.0, 0.0))
    arr = np.arange(10) * 100.0  # far apart: every request finds the service empty
    svc = FakeService()
    ol = serving.OpenLoop(svc, reqs, arr, spec_fn=identity)
    out = ol.run()
    assert ol.idle_s > 0 and all(o.late_s == pytest.approx(0.0, abs=1e-12) for o in out)
    assert all(o.queue_s == 0.0 for o in out)


def test_closed_loop_capacity():
    reqs = serving.serving_mix(400, seed=9)
    svc = FakeService()
    cap = serving.closed_loop_capacity(svc, reqs, steps=200, spec_fn=identity, depth=32)
    assert cap["converged"] > 0 and cap["cases_per_s"] == pytest.approx(cap["converged"] / cap["seconds"])


def test_request_specs_build():
    from matlab_ufvm_b200 import case
    for r in (serving.Request(0, "cavity2d", (8,), 100.0), serving.Request(1, "cavity3d", (4,), 400.0),
              serving.Request(2, "channel", (4, 2, 2), 200.0)):
        spec = serving.request_spec(r)
        assert spec.nu == pytest.approx(1.0 / r.re)
        assert spec.mesh.n_cells == r.cells
        assert spec.quirks == case.QUIRKS_CONVERGING
