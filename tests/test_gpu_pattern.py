"""tmx_pattern_ceiling on the GPU: the access pattern of each form's interior
kernel, without arithmetic, moves its bytes at a plausible rate (below the
HBM's nominal 8 TB/s, above a tenth of it) and not faster than the interior
kernel's own bytes could be moved by a plain copy of twice their size."""
import pytest

import tmixer_b200 as T

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [T.TMX_FP64, T.TMX_FP32, T.TMX_FP16])
def test_pattern_ceiling_plausible(prec):
    r = T.pattern_ceiling(prec, 1 << 21, reps=5)
    assert 800.0 < r["gbs"] < 8000.0, r
    assert r["blocks_per_sm"] in (1, 2, 4, 8)
