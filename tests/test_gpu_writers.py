"""The reference's Tecplot files written by the library from the GPU state
(tmx_write_file) against the files the compiled reference writes for the
same case and step count: Domain_Data and Data_P_V_C byte for byte; the
Pressure and MixingQuality files byte for byte against the reference's own
lines re-printed with its stock "%g" format (the test build prints those
numbers to 17 digits)."""
import math
import os

import pytest

import tmixer_b200 as T
from oracle import oracle as O
from tests.cases import to_spec
from tests.test_oracle_vs_ref import CASES, _binary

pytestmark = pytest.mark.gpu


def _g(v: float) -> str:
    """C's "%g" (which, unlike Python's, keeps the sign of a NaN)."""
    if math.isnan(v):
        return "-nan" if math.copysign(1.0, v) < 0 else "nan"
    return "%g" % v


def _line(r) -> str:
    return "\t".join(["%d" % int(r[0])] + [_g(v) for v in r[1:]]) + "\n"


def _gpu_files(case, steps, tmp_path, kinds):
    out = {}
    with T.Solver(to_spec(case)) as s:
        s.init()
        s.step(steps)
        for kind in kinds:
            p = os.path.join(tmp_path, kind)
            s.write_file(kind, p)
            with open(p, "rb") as fh:
                out[kind] = fh.read()
    return out


@pytest.mark.parametrize("name,writers", [("tiny_ref_pop", "domain"), ("pvc_rows", "pvc")])
def test_files_match_reference(gpu, tmp_path, name, writers):
    case, steps = CASES[name]
    dump, mix, _ = O.run_ref(_binary(name, case), steps, threads=2, writers=writers)
    kinds = ["domain", "pressure", "mixing"] + (["pvc"] if writers == "pvc" else [])
    got = _gpu_files(case, steps, str(tmp_path), kinds)
    assert got["domain"] == dump["files"]["Domain_Data"]
    if writers == "pvc":
        assert got["pvc"] == dump["files"]["Data_P_V_C"]

    # the stock-format lines of the reference's Pressure and MixingQuality files
    z = dump["pressure"]
    lines = ['ZONE T="PressureAlongMixingChannel" \r\n']
    lines += [_line(r) for r in z["PressureAlongMixingChannel"]]
    lines += ['ZONE T="HorizontalSectionPressure" \r\n']
    lines += [_line(r) for r in z["HorizontalSectionPressure"]]
    lines += ['ZONE T="SpecificPower"\n']
    lines += [_line(r) for r in z["SpecificPower"]]
    assert got["pressure"].decode() == "".join(lines)
    lines = ['ZONE T="Mixing Quality" \r\n', 'VARIABLES= "Y""A""B""C""IA""IB""IC"\r\n']
    lines += [_line(r) for r in mix]
    assert got["mixing"].decode() == "".join(lines)


def test_pvc_sections_outside_the_boxes_left_out(gpu, tmp_path):
    """For a mixer shorter than 600 rows the fixed sections are omitted
    (the reference would read outside its arrays); the rest is written."""
    case, steps = CASES["tiny_ref_pop"]
    got = _gpu_files(case, steps, str(tmp_path), ["pvc"])["pvc"].decode()
    assert 'ZONE T="Outlet_Z_X2' in got
    assert "MixingZ_X_600" not in got
    assert "MixingZ_X_%d(" % (case["mny"] - 1) in got


def test_driver_writes_reference_files(gpu, tmp_path):
    """tmx_run --files writes the reference's files after the steps the
    reference writes them (itr % every == 0, and Data_P_V_C at itr 100),
    named by itr, with the same bytes as the library's writer at that step."""
    import subprocess

    exe = os.path.join(os.path.dirname(T.LIB_PATH), "tmx_run")
    out = str(tmp_path)
    subprocess.run([exe, "--case", "w", "--W", "4", "--umax", "0.05", "--tauf", "0.6", "--tauc", "0.6", "--k", "1e-3",
                    "--rho", "1", "--steps", "152", "--every", "50", "--domain-every", "100", "--out", out, "--files"],
                   check=True, capture_output=True)
    names = sorted(n for n in os.listdir(out) if n.endswith(".dat"))
    want = sorted(["Data_P_V_C%d.dat" % i for i in (0, 50, 100, 150)] + ["Pressure_%d.dat" % i for i in (0, 50, 100, 150)]
                  + ["MixingQuality_%d.dat" % i for i in (0, 50, 100, 150)] + ["Domain_Data_%d.dat" % i for i in (0, 100)])
    assert names == want
    spec = T.w_layout(4, u_max=0.05, tau_f=0.6, tau_c=0.6, k=1e-3, rho=1.0)
    with T.Solver(spec) as s:
        s.init()
        s.step(101)  # itr = 100
        p = os.path.join(out, "mine")
        s.write_file("domain", p)
        with open(p, "rb") as a, open(os.path.join(out, "Domain_Data_100.dat"), "rb") as b:
            assert a.read() == b.read()
