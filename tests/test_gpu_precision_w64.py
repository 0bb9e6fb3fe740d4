"""The reduced-precision forms at the W=64 precision-form geometry (inlet
512x64x64, mixing 128x256x64: 4,194,304 nodes; u_max 0.08, tau_c 0.55,
k 5e-4, 10,000 steps) against the FP64 form on the same case: velocity and
every concentration within a relative L2 error of 1e-3, the outlet mixing
index within 1e-3, and the FP64 mass and species totals close.  tau_f is 0.6
instead of the configuration's 0.52: at 0.52 the reference's own boundary
closures diverge (the FP64 form, bit-exact with the reference, does too).

Measured (FP32 / FP16 storage): u 2.0e-4 / 2.0e-4, cA and cB 9.0e-5 /
8.8e-5, cC 3.2e-4 / 3.1e-4, mixing index 2.2e-5 / 2.8e-5, mass 5.0e-6 /
5.1e-6, species totals up to 1.2e-4 / 6.5e-5.  This case's tau_c = 0.55
(relaxation rate 1.82) is where the collision's form matters: written as
in * (1 - w) + w * feq the species errors were 5 to 15 times larger (cC
1.35e-3), written as in + w * (feq - in) they are the ones above."""
import numpy as np
import pytest

import tmixer_b200 as T

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-3  # relative L2 error of u and of each concentration field
IM_TOL = 1e-3  # absolute error of the outlet mixing index
MASS_TOL = 1e-4  # relative error of the FP64 mass total (measured 5e-6)
SPECIES_SUM_TOL = 5e-4  # relative error of the FP64 species totals (measured up to 1.2e-4)

W, STEPS = 64, 10000


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def _run(precision):
    spec = T.w_layout(W, u_max=0.08, tau_f=0.6, tau_c=0.55, k=5e-4, rho=1.0, precision=precision)
    with T.Solver(spec) as s:
        s.init()
        s.step(STEPS)
        fields = {f: np.concatenate([s.field(0, f).ravel(), s.field(1, f).ravel()]) for f in T.FIELDS}
        _, im = s.mixing()
        sums = s.sums()
    return fields, im, sums


@pytest.fixture(scope="module")
def fp64():
    return _run(T.TMX_FP64)


@pytest.mark.parametrize("precision", [T.TMX_FP32, T.TMX_FP16])
def test_w64_fields_within_tolerance(gpu, fp64, precision):
    want, im_want, sums_want = fp64
    assert sums_want[6] == 0  # the FP64 run stayed finite
    got, im, sums = _run(precision)
    u_got = np.stack([got["ux"], got["uy"], got["uz"]])
    u_want = np.stack([want["ux"], want["uy"], want["uz"]])
    assert rel_l2(u_got, u_want) <= FIELD_TOL
    for f in ("cA", "cB", "cC"):
        assert rel_l2(got[f], want[f]) <= FIELD_TOL, f
    assert np.abs(im - im_want).max() <= IM_TOL
    assert sums[6] == 0  # no non-finite values
    assert abs(sums[0] - sums_want[0]) <= MASS_TOL * abs(sums_want[0])
    for m in (1, 2, 3):
        assert abs(sums[m] - sums_want[m]) <= SPECIES_SUM_TOL * abs(sums_want[m]), m
