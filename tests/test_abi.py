"""The C-ABI library loads without a GPU, exports every entry point that
include/*.h declares, and its host-only calls (case helpers, validation,
errors) behave."""
import ctypes
import glob
import os
import re

import pytest

import tmixer_b200 as T

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[a-z_]+\s*\**\s*(tmx_[a-z0-9_]+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("tmx_create", "tmx_init", "tmx_step", "tmx_fields", "tmx_mixing", "tmx_destroy"):
        assert n in names


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports(name):
    lib = ctypes.CDLL(T.LIB_PATH)
    assert hasattr(lib, name), name


def test_abi_version():
    assert T.lib().tmx_abi_version() == T.ABI_VERSION


def test_reference_case_constants():
    c = T.reference_case()
    assert (c.inx, c.iny, c.nz, c.mnx, c.mny) == (401, 51, 51, 101, 750)
    assert (c.ia, c.ib) == (151, 251)
    assert c.tau == 0.6 and c.tau_a == (0.5 * (((2.0 * 0.6 - 1.0) / 3.0) + 1.0))
    assert c.rho0 == 3.0 and c.rho_out == 3.0 and c.rateconst == 1.0 and c.umean == 0.059761
    assert [list(r) for r in c.c_in] == [[1.0, 0.0], [0.0, 1.0], [0.0, 0.0]]
    assert c.nodes() == 401 * 51 * 51 + 101 * 750 * 51


def test_w_layout_geometry():
    c = T.w_layout(32, 0.05, 0.56, 0.6, 1e-3, 1.0)
    assert (c.inx, c.iny, c.nz, c.mnx, c.mny, c.ia, c.ib) == (256, 32, 32, 64, 128, 97, 160)
    assert c.nodes() == 524288
    assert 0.0 < c.umean < 0.05


@pytest.mark.parametrize("field,value", [("nz", 2), ("ia", 1), ("ia", 400), ("tau", 0.5), ("rho_out", 0.0),
                                         ("precision", 7)])
def test_invalid_cases_rejected(field, value):
    c = T.reference_case()
    setattr(c, field, value)
    with pytest.raises(T.TmxError) as e:
        c.check()
    assert e.value.code == -1


def test_footprint_reference_case():
    b = T.reference_case().footprint()
    assert 6.0e9 < b < 7.5e9  # about 1.34 kB per node in FP64


def test_create_without_device_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(T.TmxError) as e:
        T.Solver(T.w_layout(4, 0.05, 0.56, 0.6, 1e-3, 1.0))
    assert e.value.code == -3


@pytest.mark.parametrize("prec,nodes,reps", [(7, 1 << 20, 5), (0, 1000, 5), (2, 1 << 31, 5), (1, 1 << 20, 0)])
def test_pattern_ceiling_rejects_bad_arguments(prec, nodes, reps):
    """Argument checks come before any CUDA call, so they hold without a GPU."""
    with pytest.raises(T.TmxError) as e:
        T.pattern_ceiling(prec, nodes, reps)
    assert e.value.code == -1
