"""Reduced-precision forms (FP32; FP16 storage with FP32 arithmetic) against
the plain FP64 form on the same case: velocity and concentration fields within
a relative L2 error of 1e-3, the outlet mixing index within 1e-3, density and
the FP64 conservation sums close, and the FP16 form's stored populations,
decoded on the host, close to the FP64 populations."""
import dataclasses

import numpy as np
import pytest

import tmixer_b200 as T

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-3  # relative L2 error of u and of each concentration field
IM_TOL = 1e-3  # absolute error of the outlet mixing index
RHO_TOL = 1e-5  # relative L2 error of the density
SUM_TOL = 1e-4  # relative error of the FP64 totals of mass and species

STEPS = 3000  # species fill every row of the W=8 mixer by then


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def _run(precision, steps=STEPS, W=8):
    spec = T.w_layout(W, u_max=0.05, tau_f=0.6, tau_c=0.6, k=1e-3, rho=1.0, precision=precision)
    with T.Solver(spec) as s:
        s.init()
        s.step(steps)
        fields = {f: np.concatenate([s.field(0, f).ravel(), s.field(1, f).ravel()]) for f in T.FIELDS}
        _, im = s.mixing()
        sums = s.sums()
        pops = [s.populations(b, fld) for b in (0, 1) for fld in range(4)]
    return fields, im, sums, pops


@pytest.fixture(scope="module")
def fp64():
    return _run(T.TMX_FP64)


@pytest.mark.parametrize("precision", [T.TMX_FP32, T.TMX_FP16])
def test_fields_within_tolerance(gpu, fp64, precision):
    want, im_want, sums_want, _ = fp64
    got, im, sums, _ = _run(precision)
    u_got = np.stack([got["ux"], got["uy"], got["uz"]])
    u_want = np.stack([want["ux"], want["uy"], want["uz"]])
    assert rel_l2(u_got, u_want) <= FIELD_TOL
    for f in ("cA", "cB", "cC"):
        assert rel_l2(got[f], want[f]) <= FIELD_TOL, f
    assert rel_l2(got["rho"], want["rho"]) <= RHO_TOL
    assert np.abs(im - im_want).max() <= IM_TOL
    assert sums[6] == 0  # no non-finite values
    for m in (0, 1, 2, 3, 4):
        assert abs(sums[m] - sums_want[m]) <= SUM_TOL * abs(sums_want[m]), m


@pytest.mark.parametrize("precision", [T.TMX_FP32, T.TMX_FP16])
def test_stored_populations_close(gpu, fp64, precision):
    """The host read-back of the interleaved reduced-precision layout (and,
    for FP16, the add-back of the writer's equilibrium) returns populations
    close to the FP64 ones, direction by direction."""
    _, _, _, want = fp64
    _, _, _, got = _run(precision)
    for g, w in zip(got, want):
        assert g.shape == w.shape
        scale = np.abs(w).max(axis=tuple(range(1, w.ndim)), keepdims=True) + 1e-30
        assert (np.abs(g - w) / scale).max() <= 1e-3


@pytest.mark.parametrize("precision", [T.TMX_FP32, T.TMX_FP16])
def test_init_state_exact(gpu, precision):
    """Right after init the flow populations are w_q rho0 and the species 0,
    which every form represents exactly."""
    spec = T.w_layout(4, u_max=0.05, tau_f=0.6, tau_c=0.6, k=1e-3, rho=1.0, precision=precision)
    ref = T.w_layout(4, u_max=0.05, tau_f=0.6, tau_c=0.6, k=1e-3, rho=1.0)
    with T.Solver(spec) as s, T.Solver(ref) as r:
        s.init()
        r.init()
        for b in (0, 1):
            for fld in range(4):
                np.testing.assert_allclose(s.populations(b, fld), r.populations(b, fld), rtol=1e-6, atol=1e-7)


@pytest.mark.parametrize("precision", [T.TMX_FP32, T.TMX_FP16])
def test_device_inlet_profile(gpu, precision):
    """The reduced-precision forms compute the inlet duct series on the device
    (odd terms, sinpi); it agrees with the FP64 form's host series (the
    reference's libm bits) to 1e-12 of the profile's maximum.  (At the far
    walls the host's sin(m pi (1 +- eps)) leaves about 1e-17 where sinpi gives
    exact zeros.)"""
    spec = T.w_layout(12, u_max=0.05, tau_f=0.6, tau_c=0.6, k=1e-3, rho=1.0)
    with T.Solver(spec) as s64, T.Solver(dataclasses.replace(spec, precision=precision)) as slp:
        s64.init()
        slp.init()
        for a, b in zip(slp.inlet_profile(), s64.inlet_profile()):
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-12 * np.abs(b).max())
