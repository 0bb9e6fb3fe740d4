"""tmx_mixing_static, the mixing-quality entry point that allocates nothing:
its rows equal tmx_mixing's bit for bit on two calls in a row, at the
largest row count its fixed scratch takes, and it refuses larger cases.
Collected last so that it also runs after every other test in the process
has used the device."""
import numpy as np
import pytest

import tmixer_b200 as T
from tests.cases import GOLDEN_CASES, ref_like, to_spec
from tests.conftest import bit_equal, first_mismatch

pytestmark = pytest.mark.gpu

MAX_ROWS = 4096  # kMixStaticRows


def _same(s: T.Solver):
    want_rows, want_im = s.mixing()
    for _ in range(2):
        rows, im = s.mixing_static()
        assert bit_equal(rows, want_rows), first_mismatch(rows, want_rows)
        assert bit_equal(im, want_im)


@pytest.mark.parametrize("name", ["tiny_species", "w4"])
def test_static_rows_equal_mixing(gpu, name):
    case, steps = GOLDEN_CASES[name]
    with T.Solver(to_spec(case)) as s:
        s.init()
        _same(s)
        s.step(steps)
        _same(s)
        s.step(7)
        _same(s)


def test_static_rows_wlayout_developed(gpu):
    with T.Solver(T.w_layout(8, u_max=0.05, tau_f=0.6, tau_c=0.6, k=1e-3, rho=1.0)) as s:
        s.init()
        s.step(3000)  # long enough that every row has all three species
        want_rows, _ = s.mixing()
        assert (want_rows[:, 4:7] != 0).all()
        _same(s)


def test_static_allocates_no_device_memory(gpu):
    import torch

    case, steps = GOLDEN_CASES["tiny_ref"]
    with T.Solver(to_spec(case)) as s:
        s.init()
        s.step(steps)
        s.mixing_static()  # the first call on the device resolves the scratch
        s.sync()
        free0 = torch.cuda.mem_get_info(0)[0]
        for _ in range(3):
            s.mixing_static()
        assert torch.cuda.mem_get_info(0)[0] == free0


def test_static_at_row_limit(gpu):
    case = ref_like(8, 3, 3, 3, MAX_ROWS - 3, umean=0.02)
    with T.Solver(to_spec(case)) as s:
        s.init()
        s.step(3)
        _same(s)


def test_static_refuses_more_rows(gpu):
    case = ref_like(8, 3, 3, 3, MAX_ROWS - 2, umean=0.02)
    with T.Solver(to_spec(case)) as s:
        s.init()
        with pytest.raises(T.TmxError, match="exceeds its fixed scratch of 4096 rows"):
            s.mixing_static()
        rows, _ = s.mixing()  # the ordinary entry point still serves the case
        assert rows.shape == (MAX_ROWS + 1, 7)
