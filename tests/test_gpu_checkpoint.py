"""Checkpoint and restore: a solve saved after some steps and restored into a
new handle or a batch slot continues bit for bit as the uninterrupted solve,
in every form; checkpoints of another case or form are refused."""
import dataclasses

import pytest

import tmixer_b200 as T
from tests.cases import GOLDEN_CASES, to_spec
from tests.conftest import bit_equal, first_mismatch

pytestmark = pytest.mark.gpu

PRECISIONS = [T.TMX_FP64, T.TMX_FP32, T.TMX_FP16]


def _spec(precision, name="tiny_species"):
    return dataclasses.replace(to_spec(GOLDEN_CASES[name][0]), precision=precision)


def _fields(get):
    return {(b, f): get(b, f) for b in (0, 1) for f in T.FIELDS}


def _same(a, b):
    for key in a:
        assert bit_equal(a[key], b[key]), (key, first_mismatch(a[key], b[key]))


@pytest.mark.parametrize("precision", PRECISIONS)
def test_handle_restore_continues_bit_for_bit(gpu, precision):
    spec = _spec(precision)
    with T.Solver(spec) as s:
        s.init()
        s.step(11)
        ck = s.checkpoint()
        s.step(9)
        want = _fields(s.field)
        want_rows, _ = s.mixing()
    with T.Solver(spec) as r:  # never initialised
        r.restore(ck)
        assert r.steps_done == 11
        assert _fields(r.field) is not None
        r.step(9)
        assert r.steps_done == 20
        _same(_fields(r.field), want)
        rows, _ = r.mixing()
        assert bit_equal(rows, want_rows)


@pytest.mark.parametrize("precision", [T.TMX_FP64, T.TMX_FP16])
def test_handle_to_batch_and_back(gpu, precision):
    spec = _spec(precision)
    other = _spec(precision, "w4")
    with T.Solver(spec) as s:
        s.init()
        s.step(7)
        ck = s.checkpoint()
        s.step(6)
        want = _fields(s.field)
    with T.Batch(precision, budget=1 << 27) as B:
        B.add(other)
        B.step(3)  # the batch is at the other parity when the mixer arrives
        slot = B.restore(spec, ck)
        assert B.slot_steps(slot) == 7
        B.step(6)
        _same(_fields(lambda b, f: B.field(slot, b, f)), want)
        B.step(2)
        ck2 = B.checkpoint(slot)
    with T.Solver(spec) as r, T.Solver(spec) as s:
        r.restore(ck2)
        assert r.steps_done == 15
        s.init()
        s.step(15)
        r.step(1)
        s.step(1)
        _same(_fields(r.field), _fields(s.field))


def test_foreign_checkpoints_refused(gpu):
    with T.Solver(_spec(T.TMX_FP64)) as s:
        s.init()
        ck = s.checkpoint()
    with T.Solver(_spec(T.TMX_FP16)) as r:
        with pytest.raises(T.TmxError, match="precision"):
            r.restore(ck)
    with T.Solver(_spec(T.TMX_FP64, "w4")) as r:
        with pytest.raises(T.TmxError, match="different case|sizes"):
            r.restore(ck)
    with T.Solver(_spec(T.TMX_FP64)) as r:
        with pytest.raises(T.TmxError, match="not a checkpoint"):
            r.restore(b"x" * len(ck))
        with pytest.raises(T.TmxError, match="sizes|small"):
            r.restore(ck[:-8])
