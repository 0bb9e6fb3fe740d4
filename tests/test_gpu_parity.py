"""GPU parity: the CUDA path through the C ABI against the CPU oracle, bit
for bit (up to the sign of zero), on the fields, on all 76 populations the
state holds between steps, and on the mixing rows; and against the golden
fixtures made by the reference itself."""
import json
import os

import numpy as np
import pytest

import tmixer_b200 as T
from oracle import oracle as O
from tests.cases import GOLDEN_CASES, ORACLE_CASES, to_spec
from tests.conftest import bit_equal, first_mismatch

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ALL = dict({k: v[0] for k, v in GOLDEN_CASES.items()}, **ORACLE_CASES)

pytestmark = pytest.mark.gpu


def _compare(s: T.Solver, orc: O.Oracle, pops: bool = True):
    for b in (0, 1):
        for f in T.FIELDS:
            got, want = s.field(b, f), orc.field(b, f)
            assert bit_equal(got, want), ("field", b, f, first_mismatch(got, want))
    if pops:
        for b in (0, 1):
            for fld in range(4):
                got, want = s.populations(b, fld), orc.post_collision(b, fld)
                assert bit_equal(got, want), ("populations", b, fld, first_mismatch(got, want))
    rows, im = s.mixing()
    want = orc.mixing()
    assert bit_equal(rows, want), ("mixing", first_mismatch(rows, want))
    assert bit_equal(im, want[0, 4:7])


@pytest.mark.parametrize("name", sorted(ALL))
@pytest.mark.parametrize("steps", [1, 2, 13])
def test_step_matches_oracle(gpu, name, steps):
    case = ALL[name]
    orc = O.Oracle(case)
    with T.Solver(to_spec(case)) as s:
        s.init()
        u1, u2 = s.inlet_profile()
        o1, o2 = orc.inlet_profile()
        assert bit_equal(u1, o1) and bit_equal(u2, o2)
        s.step(steps)
        orc.step(steps)
        _compare(s, orc)
    orc.close()


@pytest.mark.parametrize("name", sorted(GOLDEN_CASES))
def test_matches_reference_fixture(gpu, name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    case = json.loads(str(g["case"]))
    steps = case.pop("steps")
    with T.Solver(to_spec(case)) as s:
        s.init()
        s.step(steps)
        for b in (0, 1):
            for f in T.FIELDS:
                got, want = s.field(b, f), g["b%d_%s" % (b, f)]
                assert bit_equal(got, want), (b, f, first_mismatch(got, want))
        rows, _ = s.mixing()
        assert bit_equal(rows, g["mixing"]), first_mismatch(rows, g["mixing"])


def test_split_steps_equal_one_call(gpu):
    case = GOLDEN_CASES["w4"][0]
    with T.Solver(to_spec(case)) as a, T.Solver(to_spec(case)) as b:
        a.init().step(17)
        b.init().step(5).step(1).step(11)
        assert a.steps_done == b.steps_done == 17
        for box in (0, 1):
            for f in T.FIELDS:
                assert bit_equal(a.field(box, f), b.field(box, f))
            for fld in range(4):
                assert bit_equal(a.populations(box, fld), b.populations(box, fld))


def test_long_run_matches_oracle(gpu):
    """Several hundred steps on the shrunk reference grid: species reach the
    outlet and the reaction is active."""
    case = GOLDEN_CASES["shrunk_ref"][0]
    orc = O.Oracle(case)
    orc.step(400)
    with T.Solver(to_spec(case)) as s:
        s.init().step(400)
        _compare(s, orc, pops=True)
        assert s.field(1, "cC").max() > 0
    orc.close()


def test_repeatable(gpu):
    case = GOLDEN_CASES["tiny_species"][0]
    outs = []
    for _ in range(2):
        with T.Solver(to_spec(case)) as s:
            s.init().step(23)
            outs.append([s.populations(b, f) for b in (0, 1) for f in range(4)])
    for x, y in zip(*outs):
        assert np.array_equal(x.view(np.uint64), y.view(np.uint64))


def test_sums_and_counts(gpu):
    case = GOLDEN_CASES["w4"][0]
    with T.Solver(to_spec(case)) as s:
        s.init().step(10)
        sums = s.sums()
        rho = np.concatenate([s.field(0, "rho").ravel(), s.field(1, "rho").ravel()])
        ca = np.concatenate([s.field(0, "cA").ravel(), s.field(1, "cA").ravel()])
        assert sums[0] == pytest.approx(rho.sum(), rel=1e-13)
        assert sums[1] == pytest.approx(ca.sum(), rel=1e-13)
        assert sums[6] == 0
        cnt = s.counts()
        assert cnt["nodes"] == case["inx"] * case["iny"] * case["nz"] + case["mnx"] * case["mny"] * case["nz"]
        assert cnt["interior"] + cnt["boundary"] == cnt["nodes"]


def test_step_timed_matches_untimed(gpu):
    case = GOLDEN_CASES["w4"][0]
    with T.Solver(to_spec(case)) as a, T.Solver(to_spec(case)) as b:
        a.init().step(6)
        b.init()
        tb, tbd, tt = b.step_timed(6)
        assert tb > 0 and tbd > 0 and tt >= tb
        for box in (0, 1):
            for fld in range(4):
                assert bit_equal(a.populations(box, fld), b.populations(box, fld))
