"""Pressure and specific power (tmx_pressure_power, the numbers of the
reference's write_Pressure_Power) on the GPU against the CPU oracle, which is
pinned bit for bit against the compiled reference
(tests/test_oracle_vs_ref.py)."""
import dataclasses

import numpy as np
import pytest

import tmixer_b200 as T
from oracle import oracle as O
from tests.cases import GOLDEN_CASES, ORACLE_CASES, to_spec
from tests.conftest import bit_equal, first_mismatch

pytestmark = pytest.mark.gpu

ALL = dict({k: v[0] for k, v in GOLDEN_CASES.items()}, **ORACLE_CASES)


@pytest.mark.parametrize("name", sorted(ALL))
def test_pressure_power_matches_oracle(gpu, name):
    case = ALL[name]
    orc = O.Oracle(case)
    orc.step(13)
    want = orc.pressure_power()
    orc.close()
    with T.Solver(to_spec(case)) as s:
        s.init()
        s.step(13)
        got = s.pressure_power()
    for g, w, what in zip(got, want, ("rows", "sections", "power", "units")):
        assert bit_equal(g, w), (what, first_mismatch(g, w))


def test_pressure_power_reduced_precision(gpu):
    """The FP16-storage form's pressure profile stays within 1e-4 relative of
    the FP64 one after 2000 steps of a W=8 mixer."""
    spec = T.w_layout(8, u_max=0.05, tau_f=0.6, tau_c=0.6, k=1e-3, rho=1.0)
    out = []
    for p in (T.TMX_FP64, T.TMX_FP16):
        with T.Solver(dataclasses.replace(spec, precision=p)) as s:
            s.init()
            s.step(2000)
            out.append(s.pressure_power())
    (r64, x64, w64, _), (r16, x16, w16, _) = out
    assert np.allclose(r16[:, 1], r64[:, 1], rtol=1e-4)
    assert np.allclose(x16[:, 1], x64[:, 1], rtol=1e-4)
    assert np.allclose(w16[:, 4], w64[:, 4], rtol=2e-2, atol=1e-9)
