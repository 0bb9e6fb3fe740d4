"""Batched engine: every mixer of a batch evolves exactly as it does alone
(bit for bit against a single-mixer handle of the same precision), whatever
else shares the batch, whenever it was admitted, and across removals,
back-fills, retuning and admission by footprint."""
import dataclasses

import numpy as np
import pytest

import tmixer_b200 as T
from tests.cases import GOLDEN_CASES, ORACLE_CASES, to_spec
from tests.conftest import bit_equal, first_mismatch

pytestmark = pytest.mark.gpu

PRECISIONS = [T.TMX_FP64, T.TMX_FP32, T.TMX_FP16]


def _specs(precision):
    cases = [GOLDEN_CASES["tiny_species"][0], GOLDEN_CASES["w4"][0], ORACLE_CASES["odd_ia"],
             GOLDEN_CASES["tiny_ref"][0]]
    return [dataclasses.replace(to_spec(c), precision=precision) for c in cases]


def _alone(spec, steps):
    with T.Solver(spec) as s:
        s.init()
        s.step(steps)
        fields = {(b, f): s.field(b, f) for b in (0, 1) for f in T.FIELDS}
        rows, _ = s.mixing()
    return fields, rows[0, 4:7].copy()


def _same(batch, slot, want, steps):
    fields, im = want
    assert batch.slot_steps(slot) == steps
    for (b, f), w in fields.items():
        got = batch.field(slot, b, f)
        assert bit_equal(got, w), (slot, b, f, first_mismatch(got, w))
    got_im = batch.outlet_im([slot])[0]
    assert bit_equal(got_im, im), (got_im, im)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_batch_equals_alone(gpu, precision):
    specs = _specs(precision)
    with T.Batch(precision, budget=1 << 28) as B:
        slots = [B.add(s) for s in specs]
        B.step(23)
        for slot, spec in zip(slots, specs):
            _same(B, slot, _alone(spec, 23), 23)


@pytest.mark.parametrize("precision", [T.TMX_FP64, T.TMX_FP16])
def test_admitted_later_same_as_alone(gpu, precision):
    """A mixer admitted after the others have taken an odd number of steps
    (the other parity of the batch's buffers) still matches its solo run."""
    specs = _specs(precision)
    with T.Batch(precision, budget=1 << 28) as B:
        first = [B.add(s) for s in specs[:2]]
        B.step(7)
        late = B.add(specs[2])
        B.step(12)
        _same(B, late, _alone(specs[2], 12), 12)
        for slot, spec in zip(first, specs[:2]):
            _same(B, slot, _alone(spec, 19), 19)


def test_remove_and_backfill(gpu):
    specs = _specs(T.TMX_FP16)
    with T.Batch(T.TMX_FP16, budget=1 << 28) as B:
        a, b, c = (B.add(s) for s in specs[:3])
        B.step(5)
        B.remove(b)
        d = B.add(specs[3])  # reuses the freed slot and, first fit, its range
        assert d == b
        B.step(9)
        _same(B, a, _alone(specs[0], 14), 14)
        _same(B, c, _alone(specs[2], 14), 14)
        _same(B, d, _alone(specs[3], 9), 9)


def test_admission_by_footprint(gpu):
    spec = _specs(T.TMX_FP16)[1]
    fp = T.Batch.footprint(spec)
    with T.Batch(T.TMX_FP16, budget=2 * fp + 1024) as B:
        s0 = B.add(spec)
        B.add(spec)
        with pytest.raises(T.TmxError, match="batch budget"):
            B.add(spec)
        B.remove(s0)
        B.add(spec)
        assert len(B.slots()) == 2


def test_tune_restarts_mixers(gpu):
    specs = _specs(T.TMX_FP16)
    with T.Batch(T.TMX_FP16, budget=1 << 28) as B:
        slots = [B.add(s) for s in specs]
        best = B.tune(steps_per_trial=3)
        assert best["kernel"] in T.SHAPE_NAMES.values()
        assert best["threads"] in (128, 256, 512) and best["cells"] % best["threads"] == 0
        shape = B.shape()
        assert all(shape[k] == best[k] for k in ("kernel", "threads", "cells", "zchunk", "boundary_blocks_per_sm",
                                                 "interior_after_boundary"))
        assert shape["boundary_blocks_per_sm"] >= 1
        B.step(11)
        for slot, spec in zip(slots, specs):
            _same(B, slot, _alone(spec, 11), 11)


@pytest.mark.parametrize("precision,bps,after", [(T.TMX_FP16, 1, False), (T.TMX_FP16, 0, True),
                                                 (T.TMX_FP64, 2, False)])
def test_boundary_grids_agree(gpu, precision, bps, after):
    """A smaller persistent grid of the boundary kernels (each block then
    takes more 32-entry chunks, of several mixers) gives each mixer its solo
    run's bits."""
    specs = _specs(precision)
    with T.Batch(precision, budget=1 << 28) as B:
        B.set_boundary(bps, after)
        shape = B.shape()
        assert shape["interior_after_boundary"] == (after or precision == T.TMX_FP64)
        if bps:
            assert shape["boundary_blocks_per_sm"] == bps
        slots = [B.add(s) for s in specs]
        B.step(6)
        for slot, spec in zip(slots, specs):
            _same(B, slot, _alone(spec, 6), 6)
        B.set_boundary(0)
        assert B.shape()["boundary_blocks_per_sm"] > max(bps, 1)


def test_step_timed_agrees(gpu):
    """Timed steps (kernels one after another, no graph) give each mixer its
    solo run's bits and count as steps."""
    specs = _specs(T.TMX_FP16)
    with T.Batch(T.TMX_FP16, budget=1 << 28) as B:
        B.set_sweep(T.SHAPE_SWEEP4, 4)
        slots = [B.add(s) for s in specs]
        B.step(3)
        ti, tb, tt = B.step_timed(4)
        assert ti > 0 and tb > 0 and tt >= ti
        B.step(1)
        for slot, spec in zip(slots, specs):
            assert B.slot_steps(slot) == 8
            _same(B, slot, _alone(spec, 8), 8)


@pytest.mark.parametrize("threads,cells", [(128, 1024), (512, 8192)])
def test_launch_shapes_agree(gpu, threads, cells):
    specs = _specs(T.TMX_FP32)
    with T.Batch(T.TMX_FP32, budget=1 << 28) as B:
        B.set_shape(threads, cells)
        slots = [B.add(s) for s in specs]
        B.step(6)
        for slot, spec in zip(slots, specs):
            _same(B, slot, _alone(spec, 6), 6)


def test_wrong_precision_rejected(gpu):
    with T.Batch(T.TMX_FP16, budget=1 << 26) as B:
        with pytest.raises(T.TmxError, match="precision"):
            B.add(_specs(T.TMX_FP32)[0])


@pytest.mark.parametrize("kind,zchunk", [(T.SHAPE_SWEEP8, 3), (T.SHAPE_SWEEP4, 1), (T.SHAPE_SWEEP8, 64),
                                         (T.SHAPE_SWEEP4, 16)])
def test_sweep_shapes_agree(gpu, kind, zchunk):
    """The FP16 form's sweep interior kernel in a batch (tiles of every mixer
    in one list) gives each mixer its solo run's bits."""
    specs = _specs(T.TMX_FP16)
    with T.Batch(T.TMX_FP16, budget=1 << 28) as B:
        B.set_sweep(kind, zchunk)
        slots = [B.add(s) for s in specs]
        B.step(6)
        late = B.add(specs[1])
        B.step(5)
        for slot, spec in zip(slots, specs):
            _same(B, slot, _alone(spec, 11), 11)
        _same(B, late, _alone(specs[1], 5), 5)
        assert B.shape()["kernel"] == T.SHAPE_NAMES[kind]
        B.set_shape(256, 4096)
        assert B.shape()["kernel"] == "flat"
