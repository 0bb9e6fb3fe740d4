"""The served form's request loop (tmx_serve_with, the same C++ scheduler that
tmx_serve runs over a GPU batch) against a fake engine on the CPU: admission
in arrival order under the memory budget, back-fill of retired ranges,
retirement on convergence of the outlet mixing index or at max_steps, idling
until arrivals, and the summary statistics."""
import math

import numpy as np
import pytest

import tmixer_b200 as T

CHECK = 100


def spec(W: int, tau_steps: float):
    # the fake engine reads the convergence time constant from rateconst
    s = T.w_layout(W, u_max=0.05, tau_f=0.6, tau_c=0.6, k=1e-3, rho=1.0)
    s.rateconst = float(tau_steps)
    return s


class FakeEngine:
    """Memory accounting like the batch arena (bytes = 100 per node), a clock
    that advances with the work of every step, and an outlet index that
    approaches its limit as 1 - exp(-steps / tau)."""

    def __init__(self, capacity: int, nodes_per_second: float = 1e8):
        self.cap = capacity
        self.rate = nodes_per_second
        self.clock = 0.0
        self.used = 0
        self.slots = {}
        self.admissions = []  # (time, slot, spec)
        self.removals = []
        self.max_used = 0

    def footprint(self, s):
        return s.nodes() * 100

    def capacity(self):
        return self.cap

    def add(self, s):
        fp = self.footprint(s)
        if self.used + fp > self.cap:
            return None
        slot = min(set(range(len(self.slots) + 1)) - set(self.slots))
        self.slots[slot] = dict(spec=s, steps=0, fp=fp)
        self.used += fp
        self.max_used = max(self.max_used, self.used)
        self.admissions.append((self.clock, slot, s))
        return slot

    def remove(self, slot):
        e = self.slots.pop(slot)
        self.used -= e["fp"]
        self.removals.append((self.clock, slot))

    def step(self, n):
        work = sum(e["spec"].nodes() for e in self.slots.values())
        self.clock += n * work / self.rate
        for e in self.slots.values():
            e["steps"] += n

    @staticmethod
    def im(tau, steps):
        # tau < 0: the species never reach the outlet (index 0, undefined)
        if tau < 0:
            return [0.0, 0.0, 0.0]
        v = 1.0 - math.exp(-steps / tau)
        return [0.5 * v, 0.5 * v, 0.9 * v]

    def outlet_im(self, slots):
        return [self.im(self.slots[s]["spec"].rateconst, self.slots[s]["steps"]) for s in slots]

    def now(self):
        return self.clock

    def wait_until(self, t):
        self.clock = max(self.clock, t)


def expected_steps(tau, window, tol, max_steps):
    s = CHECK
    while True:
        if s >= window:
            hist = [FakeEngine.im(tau, t) for t in range(s - window, s + 1, CHECK)]
            a, b = hist[-1], hist[0]
            if all(v != 0 for h in hist for v in h) and all(abs(x - y) < tol for x, y in zip(a, b)):
                return s, "converged"
        if s >= max_steps:
            return s, "max_steps"
        s += CHECK


def test_convergence_and_max_steps():
    reqs = [T.Request(spec(4, 300.0), 0.0, 50000, 500, 1e-6), T.Request(spec(4, 900.0), 0.0, 50000, 500, 1e-6),
            T.Request(spec(4, 5000.0), 0.0, 3000, 500, 1e-6)]
    eng = FakeEngine(capacity=10**9)
    res, summ = T.serve_with(eng, reqs, check_every=CHECK)
    for q, r in zip(reqs, res):
        steps, status = expected_steps(q.spec.rateconst, q.window, q.tol, q.max_steps)
        assert (r["steps"], r["status"]) == (steps, status)
        want = FakeEngine.im(q.spec.rateconst, steps)
        assert r["outlet_im"] == pytest.approx(want, rel=0, abs=0)
    assert summ["lattice_updates"] == sum(q.spec.nodes() * r["steps"] for q, r in zip(reqs, res))
    assert not eng.slots  # every mixer was removed


def test_admission_order_budget_and_backfill():
    s = spec(4, 400.0)
    fp = s.nodes() * 100
    reqs = [T.Request(spec(4, 400.0 + 100 * i), 0.001 * i, 50000, 500, 1e-6) for i in range(6)]
    eng = FakeEngine(capacity=2 * fp + 10)  # room for two mixers at a time
    res, summ = T.serve_with(eng, reqs, check_every=CHECK)
    assert eng.max_used <= eng.cap
    assert summ["max_active"] == 2
    # admitted in arrival order
    adm = [r["admitted"] for r in res]
    assert adm == sorted(adm)
    assert [a[2].rateconst for a in eng.admissions] == [q.spec.rateconst for q in reqs]
    # each request after the first two fills the range of a retirement at that very check
    fin = sorted(r["finished"] for r in res)
    for r in res[2:]:
        assert r["admitted"] in fin
    assert all(r["status"] == "converged" for r in res)


def test_idle_until_arrival_and_percentiles():
    reqs = [T.Request(spec(4, 300.0), 0.0, 50000, 500, 1e-6), T.Request(spec(4, 300.0), 5.0, 50000, 500, 1e-6),
            T.Request(spec(6, 600.0), 9.0, 50000, 500, 1e-6)]
    eng = FakeEngine(capacity=10**9, nodes_per_second=1e7)
    res, summ = T.serve_with(eng, reqs, check_every=CHECK)
    for q, r in zip(reqs, res):
        assert r["admitted"] >= q.arrival
    assert res[1]["admitted"] == pytest.approx(5.0)  # the loop idled until it arrived
    tts = sorted(r["time_to_solution"] for r in res)
    assert summ["p50_s"] == tts[1] and summ["p99_s"] == tts[2]
    assert summ["makespan_s"] == max(r["finished"] for r in res)
    assert summ["mlups"] == pytest.approx(summ["lattice_updates"] / summ["makespan_s"] / 1e6)


def test_too_large_rejected_others_served():
    small, big = spec(4, 300.0), spec(8, 300.0)
    eng = FakeEngine(capacity=small.nodes() * 100 + 5)
    res, _ = T.serve_with(eng, [T.Request(big, 0.0), T.Request(small, 0.0, window=500, tol=1e-6)],
                          check_every=CHECK)
    assert res[0]["status"] == "too large for the budget"
    assert res[1]["status"] == "converged"


def test_max_active_limit():
    reqs = [T.Request(spec(4, 300.0 + 50 * i), 0.0) for i in range(5)]
    eng = FakeEngine(capacity=10**9)
    _, summ = T.serve_with(eng, reqs, check_every=CHECK, max_active=2)
    assert summ["max_active"] == 2


def test_bad_window_rejected():
    eng = FakeEngine(capacity=10**9)
    with pytest.raises(T.TmxError, match="window"):
        T.serve_with(eng, [T.Request(spec(4, 300.0), 0.0, 1000, 250, 1e-6)], check_every=CHECK)


def test_undefined_index_never_converges():
    """An outlet index of 0 (species not yet at the outlet) does not count as
    converged, however constant it is."""
    eng = FakeEngine(capacity=10**9)
    res, _ = T.serve_with(eng, [T.Request(spec(4, -1.0), 0.0, 2000, 500, 1e-6)], check_every=CHECK)
    assert (res[0]["status"], res[0]["steps"]) == ("max_steps", 2000)


class SickEngine(FakeEngine):
    """A fake engine whose mixers of tau == 777 turn non-finite after 300
    steps."""

    def health(self, slots):
        return [int(self.slots[s]["spec"].rateconst == 777.0 and self.slots[s]["steps"] >= 300) for s in slots]


def test_non_finite_mixer_retired_and_backfilled():
    s = spec(4, 400.0)
    reqs = [T.Request(spec(4, 777.0), 0.0, 50000, 500, 1e-6), T.Request(spec(4, 400.0), 0.0, 50000, 500, 1e-6)]
    eng = SickEngine(capacity=s.nodes() * 100 + 10)  # one mixer at a time
    res, summ = T.serve_with(eng, reqs, check_every=CHECK)
    assert (res[0]["status"], res[0]["steps"]) == ("non-finite", 300)
    assert res[1]["status"] == "converged"
    assert res[1]["admitted"] == res[0]["finished"]  # back-filled at once
    # a diverged solve has no time to solution
    assert summ["p99_s"] == res[1]["time_to_solution"]


class PickyEngine(FakeEngine):
    """A fake engine that refuses (TMX_E_INVALID) every case of width 6."""

    def add(self, s):
        if s.iny == 6:
            return -1
        return super().add(s)


def test_refused_case_fails_alone():
    """A request the engine cannot take (an invalid case, a precision other
    than the batch's) is finished with the engine's error code; the loop goes
    on with the others."""
    reqs = [T.Request(spec(4, 300.0), 0.0), T.Request(spec(6, 300.0), 0.0), T.Request(spec(4, 400.0), 0.0)]
    eng = PickyEngine(capacity=10**9)
    res, summ = T.serve_with(eng, reqs, check_every=CHECK)
    assert res[1]["status"] == -1 and res[1]["steps"] == 0
    assert res[0]["status"] == "converged" and res[2]["status"] == "converged"
    assert not eng.slots


class FailingEngine(FakeEngine):
    """A fake engine whose step fails once the clock passes 1e-3 s."""

    def step(self, n):
        if self.clock > 1e-3:
            raise RuntimeError("device lost")
        super().step(n)


def test_engine_error_releases_active_slots():
    """An error of the engine's step ends the loop with that error, after
    every admitted mixer has been removed from the engine."""
    reqs = [T.Request(spec(4, 300.0 + 10 * i), 0.0) for i in range(3)]
    eng = FailingEngine(capacity=10**9)
    with pytest.raises(RuntimeError, match="device lost"):
        T.serve_with(eng, reqs, check_every=CHECK)
    assert len(eng.admissions) == 3 and not eng.slots
