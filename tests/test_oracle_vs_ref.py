"""The oracle against the reference binary itself, including all 76
post-step populations of every node, on cases the fixtures do not cover.
Runs where the reference binaries exist (built from the reference source by
oracle/build_ref.py; prebuilt binaries travel with the repository)."""
import glob
import os

import pytest

from oracle import build_ref, oracle as O
from tests.cases import GOLDEN_CASES, ref_params, ref_like, w_like
from tests.conftest import bit_equal, first_mismatch

CASES = {
    "tiny_ref_pop": (GOLDEN_CASES["tiny_ref"][0], 9),
    # long and thin: the reference's fixed section rows 600, mny-1 and
    # 775-mny = 5 of write_Data_P_V_C all lie inside its boxes
    "pvc_rows": (ref_like(9, 8, 3, 3, 770, umean=0.02), 6),
    "w3_pop": (w_like(3, umean=0.04, tau=0.58, tau_c=0.7, k=0.8, rho=1.2), 25),
    "species_pop": (GOLDEN_CASES["tiny_species"][0], 17),
    # the opening (ia = 2 .. ib = 6) next to both inlet faces: the junction
    # edges DD' and CC' share their rows with the inlet faces' neighbours
    "wide_opening": (ref_like(7, 4, 4, 5, 5, umean=0.03), 12),
}


def _binary(name, case):
    path = build_ref.binary_path("t_" + name, ref_params(case))
    if os.path.exists(path):
        return path
    if os.path.exists(build_ref.REF_SRC):
        return build_ref.build("t_" + name, ref_params(case))
    pytest.skip("reference source and prebuilt reference binary both absent")


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_populations_match_reference(name):
    case, steps = CASES[name]
    dump, mix, _ = O.run_ref(_binary(name, case), steps, with_pops=True, threads=2)
    orc = O.Oracle(case)
    orc.step(steps)
    for b in (0, 1):
        for f in O.FIELDS:
            assert bit_equal(orc.field(b, f), dump[(b, f)]), (b, f, first_mismatch(orc.field(b, f), dump[(b, f)]))
        for fld in range(4):
            got, want = orc.pops(b, fld), dump[(b, "pops", fld)]
            assert bit_equal(got, want), (b, fld, first_mismatch(got, want))
    assert bit_equal(orc.mixing(), mix)
    orc.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_pressure_power_matches_reference(name):
    """write_Pressure_Power's numbers (Tmixer.cpp:9866-10027, printed to 17
    digits by the patched build): the lattice values bit for bit, and the
    values the reference multiplies by its unit factors too."""
    case, steps = CASES[name]
    dump, _, _ = O.run_ref(_binary(name, case), steps, threads=2)
    ref = dump["pressure"]
    orc = O.Oracle(case)
    orc.step(steps)
    prow, px, pw, (p0, pw0) = orc.pressure_power()
    orc.close()
    rows = ref["PressureAlongMixingChannel"]
    assert bit_equal(rows[:, 0], prow[:, 0]) and bit_equal(rows[:, 1], prow[:, 1])
    assert bit_equal(rows[:, 2], prow[:, 1] * p0) and bit_equal(rows[:, 3], prow[:, 2] * p0)
    hor = ref["HorizontalSectionPressure"]
    assert bit_equal(hor[:, 0], px[:, 0]) and bit_equal(hor[:, 1], px[:, 1]) and bit_equal(hor[:, 2], px[:, 1] * p0)
    pwr = ref["SpecificPower"]
    assert bit_equal(pwr[:, 0], pw[:, 0]) and bit_equal(pwr[:, 1], pw[:, 1])
    assert bit_equal(pwr[:, 2], pw[:, 1] * pw0) and bit_equal(pwr[:, 3], pw[:, 2] * pw0)
