"""Served form on the GPU: continuous batching gives each request the same
result as running it alone (steps taken, stop reason and outlet mixing
index, bit for bit), whether its neighbours arrive before, with or after it
and whether the budget lets all of them in at once or only two."""
import dataclasses

import numpy as np
import pytest

import tmixer_b200 as T
from tests.cases import GOLDEN_CASES, ORACLE_CASES, to_spec

pytestmark = pytest.mark.gpu


def _requests(precision=T.TMX_FP16):
    cases = [GOLDEN_CASES["tiny_species"][0], GOLDEN_CASES["w4"][0], ORACLE_CASES["odd_ia"],
             GOLDEN_CASES["tiny_ref"][0]]
    specs = [dataclasses.replace(to_spec(c), precision=precision) for c in cases]
    arrivals = [0.0, 0.0, 0.05, 0.1]
    return [T.Request(s, a, max_steps=1200, window=300, tol=1e-7) for s, a in zip(specs, arrivals)]


def _alone(q):
    with T.Batch(q.spec.precision, budget=1 << 27) as B:
        res, _ = T.serve(B, [dataclasses.replace(q, arrival=0.0)], check_every=100)
    return res[0]


@pytest.mark.parametrize("budget_mixers", [None, 2])
def test_same_alone_and_in_mix(gpu, budget_mixers):
    reqs = _requests()
    budget = 1 << 27
    if budget_mixers:
        budget = max(T.Batch.footprint(q.spec) for q in reqs) * budget_mixers + 4096
    with T.Batch(T.TMX_FP16, budget=budget) as B:
        mixed, summ = T.serve(B, reqs, check_every=100)
    assert summ["max_active"] >= 2
    if budget_mixers:
        assert summ["max_active"] <= budget_mixers
    for q, got in zip(reqs, mixed):
        want = _alone(q)
        assert got["status"] == want["status"] and got["steps"] == want["steps"]
        assert got["outlet_im"] == want["outlet_im"]  # exact
        assert got["admitted"] >= q.arrival


def test_served_outlet_index_matches_solver(gpu):
    """The retired outlet index is the one a single-mixer handle reports after
    the same number of steps."""
    q = _requests(T.TMX_FP32)[0]
    r = _alone(q)
    with T.Solver(q.spec) as s:
        s.init()
        s.step(r["steps"])
        _, im = s.mixing()
    assert list(im) == r["outlet_im"]


def test_health_flags_non_finite_mixers(gpu):
    """A mixer restored from a checkpoint whose populations were overwritten
    with NaN is flagged by the device health check after a step; its
    neighbour in the batch is not, and keeps its exact result."""
    healthy, sick = _requests()[0].spec, _requests()[1].spec
    with T.Solver(sick) as s:
        s.init()
        s.step(5)
        ck = bytearray(s.checkpoint())
    ck[1000:1256] = b"\x7e" * 256  # FP16 0x7E7E: NaN
    with T.Batch(T.TMX_FP16, budget=1 << 27) as B:
        a = B.add(healthy)
        b = B.restore(sick, bytes(ck))
        B.step(2)
        assert B.health([a, b]) == [0, 1]
        B.step(3)
        with T.Solver(healthy) as s:
            s.init()
            s.step(5)
            want = s.field(1, "cA")
        assert np.array_equal(B.field(a, 1, "cA"), want)
