"""The reference's own hard-coded case at full size (inlet 401x51x51 +
mixing 101x750x51, 4.9M nodes): after 100 and after 1,000 steps every field
of both boxes and the mixing rows equal the compiled reference's, bit for bit
(digests in tests/golden/reference_case_<steps>.json, made by
tests/golden/make_golden.py --full <steps>), and repeated runs of every form
give the same bits."""
import json
import os

import numpy as np
import pytest

import tmixer_b200 as T
from tests.golden.make_golden import digest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_case_%d.json")


@pytest.mark.parametrize("steps", [100, 1000])
def test_reference_case_bit_exact(gpu, steps):
    with open(GOLDEN % steps) as fh:
        want = json.load(fh)
    assert want["steps"] == steps
    with T.Solver(T.reference_case()) as s:
        s.init()
        s.step(want["steps"])
        for b in (0, 1):
            for f in T.FIELDS:
                assert digest(s.field(b, f)) == want["fields"]["b%d_%s" % (b, f)], (b, f)
        rows, _ = s.mixing()
        assert rows.shape[0] == want["mixing_rows"]
        assert digest(rows) == want["mixing"]


@pytest.mark.parametrize("precision", [T.TMX_FP64, T.TMX_FP32, T.TMX_FP16])
def test_runs_repeat_bit_for_bit(gpu, precision):
    spec = T.w_layout(16, u_max=0.05, tau_f=0.6, tau_c=0.6, k=1e-3, rho=1.0, precision=precision)
    out = []
    for _ in range(2):
        with T.Solver(spec) as s:
            s.init()
            s.step(300)
            out.append([s.field(b, f) for b in (0, 1) for f in T.FIELDS] + [s.populations(1, 2)])
    for a, b in zip(*out):
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
