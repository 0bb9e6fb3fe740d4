"""The CPU oracle against the golden fixtures made by running the reference
itself (tests/golden/make_golden.py): bit-exact fields and mixing rows."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.cases import GOLDEN_CASES
from tests.conftest import bit_equal, first_mismatch

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module", autouse=True)
def _built():
    O.build()


@pytest.mark.parametrize("name", sorted(GOLDEN_CASES))
def test_oracle_matches_reference_fixture(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    case = json.loads(str(g["case"]))
    steps = case.pop("steps")
    assert case == dict(GOLDEN_CASES[name][0]), "fixture made for a different case; regenerate"
    orc = O.Oracle(case)
    orc.step(steps)
    for b in (0, 1):
        for f in O.FIELDS:
            got, want = orc.field(b, f), g["b%d_%s" % (b, f)]
            assert bit_equal(got, want), (b, f, first_mismatch(got, want))
    assert bit_equal(orc.mixing(), g["mixing"]), first_mismatch(orc.mixing(), g["mixing"])
    orc.close()


def test_fixtures_are_nontrivial():
    """The fixtures must exercise the reaction and both inlets."""
    g = np.load(os.path.join(GOLDEN, "shrunk_ref.npz"))
    assert g["b1_cC"].max() > 0
    assert g["b0_cA"].max() > 0.5 and g["b0_cB"].max() > 0.5
    assert np.isfinite(g["b1_rho"]).all()
