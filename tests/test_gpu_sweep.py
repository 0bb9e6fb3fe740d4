"""The FP16 form's tiled interior kernels (TMX_SHAPE_SWEEP8 / SWEEP4: tiles of
32 x 8 or 32 x 4 nodes walked through z, the writers' moment records staged in
shared memory) give the flat kernel's results bit for bit: every population,
moment-derived field and mixing row, on geometries whose boxes are not
multiples of the tile (ragged x and y tiles), with the opening next to the
inlet faces, and with z-chunks of one plane up to the whole box."""
import numpy as np
import pytest

import tmixer_b200 as T
from tests.cases import GOLDEN_CASES, ORACLE_CASES, to_spec

pytestmark = pytest.mark.gpu


def _case(name):
    if name in GOLDEN_CASES:
        return to_spec(GOLDEN_CASES[name][0])
    return to_spec(ORACLE_CASES[name])


def _state(spec, shape, zchunk, steps):
    with T.Solver(spec) as s:
        if shape is not None:  # None: the handle's default shape
            s.set_shape(shape, zchunk)
        s.init()
        s.step(steps)
        fields = [s.field(b, f) for b in (0, 1) for f in T.FIELDS]
        pops = [s.populations(b, fld) for b in (0, 1) for fld in range(4)]
        rows, _ = s.mixing()
    return fields + pops + [rows]


def _same(a, b):
    return all(np.array_equal(x.view(np.uint64), y.view(np.uint64)) for x, y in zip(a, b))


CASES = [("w24", None), ("tiny_species", None), ("wide_opening", None), ("odd_ia", None), ("w8", None)]


def _spec(name):
    if name.startswith("w") and name[1:].isdigit():
        return T.w_layout(int(name[1:]), u_max=0.05, tau_f=0.6, tau_c=0.6, k=1e-3, rho=1.0, precision=T.TMX_FP16)
    s = _case(name)
    s.precision = T.TMX_FP16
    return s


@pytest.mark.parametrize("name", [c[0] for c in CASES])
def test_sweep_equals_flat(gpu, name):
    spec = _spec(name)
    steps = 25
    want = _state(spec, T.SHAPE_FLAT, 8, steps)
    for shape, zchunk in ((None, 0), (T.SHAPE_SWEEP8, 8), (T.SHAPE_SWEEP4, 3), (T.SHAPE_SWEEP8, 1),
                          (T.SHAPE_SWEEP4, 1000)):
        got = _state(spec, shape, zchunk, steps)
        assert _same(got, want), (name, shape, zchunk)


def test_sweep_shape_rejected_outside_fp16(gpu):
    spec = T.w_layout(4, u_max=0.05, tau_f=0.6, tau_c=0.6, k=1e-3, rho=1.0, precision=T.TMX_FP32)
    with T.Solver(spec) as s:
        with pytest.raises(T.TmxError):
            s.set_shape(T.SHAPE_SWEEP8, 8)
        s.set_shape(T.SHAPE_FLAT, 8)
