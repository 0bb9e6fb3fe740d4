"""ctypes wrapper of the CPU oracle (oracle/tmx_oracle.c) and of the compiled
reference harness (oracle/_ref).  Test infrastructure only: imported by tests/,
by ``__graft_entry__.smoke()`` and by the CPU-baseline leg of ``bench.py``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "tmx_oracle.c")
LIB = os.path.join(HERE, "libtmx_oracle.so")

FIELDS = ("rho", "ux", "uy", "uz", "cA", "cB", "cC")


class OrcParams(ctypes.Structure):
    _fields_ = [("inx", ctypes.c_int), ("iny", ctypes.c_int), ("nz", ctypes.c_int),
                ("mnx", ctypes.c_int), ("mny", ctypes.c_int), ("ia", ctypes.c_int),
                ("tau", ctypes.c_double), ("taua", ctypes.c_double), ("taub", ctypes.c_double),
                ("taup", ctypes.c_double), ("rho0", ctypes.c_double), ("rho_out", ctypes.c_double),
                ("c0", ctypes.c_double), ("cin", (ctypes.c_double * 2) * 3),
                ("rateconst", ctypes.c_double), ("umean", ctypes.c_double)]


def build(force: bool = False) -> str:
    """Compile the oracle shared library (gcc, no FMA contraction)."""
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        tmp = LIB + ".tmp"
        subprocess.run(["gcc", "-O2", "-std=c11", "-fopenmp", "-ffp-contract=off", "-shared", "-fPIC",
                        "-o", tmp, SRC, "-lm"], check=True)
        os.replace(tmp, LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.POINTER(OrcParams)]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_init.argtypes = [ctypes.c_void_p]
        L.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_fields.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        L.orc_pops.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        L.orc_mixing.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_pressure_power.argtypes = [ctypes.c_void_p] * 5
        L.orc_inlet_profile.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_collide_preview.argtypes = [ctypes.c_void_p]
        L.orc_fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        _lib = L
    return _lib


def params_from_case(case: dict) -> OrcParams:
    """``case`` uses the keys of tmixer_b200.CaseSpec (plain dict)."""
    p = OrcParams()
    for k in ("inx", "iny", "nz", "mnx", "mny", "ia"):
        setattr(p, k, int(case[k]))
    for k in ("tau", "taua", "taub", "taup", "rho0", "rho_out", "c0", "rateconst", "umean"):
        setattr(p, k, float(case[k]))
    cin = case["cin"]
    for s in range(3):
        for n in range(2):
            p.cin[s][n] = float(cin[s][n])
    return p


class Oracle:
    """One oracle run of a case; mirrors the reference's phase order."""

    def __init__(self, case: dict):
        self.case = dict(case)
        self._p = params_from_case(case)
        self._h = lib().orc_create(ctypes.byref(self._p))
        if not self._h:
            raise MemoryError("oracle allocation failed")
        lib().orc_init(self._h)

    def step(self, n: int = 1) -> None:
        lib().orc_step(self._h, int(n))

    def box_shape(self, box: int):
        c = self.case
        return (c["inx"], c["iny"], c["nz"]) if box == 0 else (c["mnx"], c["mny"], c["nz"])

    def field(self, box: int, name: str) -> np.ndarray:
        out = np.empty(self.box_shape(box), dtype=np.float64)
        lib().orc_fields(self._h, box, FIELDS.index(name), out.ctypes.data)
        return out

    def pops(self, box: int, fld: int) -> np.ndarray:
        out = np.empty((19,) + self.box_shape(box), dtype=np.float64)
        for q in range(19):
            lib().orc_pops(self._h, box, fld, q, out[q].ctypes.data)
        return out

    def post_collision(self, box: int, fld: int) -> np.ndarray:
        """The populations the next step streams (what the GPU state holds
        between steps), shape (19, nx, ny, nz)."""
        lib().orc_collide_preview(self._h)
        out = np.empty((19,) + self.box_shape(box), dtype=np.float64)
        for q in range(19):
            lib().orc_fn(self._h, box, fld, q, out[q].ctypes.data)
        return out

    def mixing(self) -> np.ndarray:
        rows = np.empty((self.case["mny"] + self.case["iny"], 7), dtype=np.float64)
        lib().orc_mixing(self._h, rows.ctypes.data)
        return rows

    def pressure_power(self):
        """(pressure rows (mny+iny, 3), cross-section pressures (inx, 2),
        power rows (mny-2, 5), units (P0, Pw0)) as orc_pressure_power."""
        c = self.case
        prow = np.empty((c["mny"] + c["iny"], 3))
        px = np.empty((c["inx"], 2))
        pw = np.empty((c["mny"] - 2, 5))
        units = np.empty(2)
        lib().orc_pressure_power(self._h, prow.ctypes.data, px.ctypes.data, pw.ctypes.data, units.ctypes.data)
        return prow, px, pw, units

    def inlet_profile(self):
        n = (self.case["iny"] + 3, self.case["nz"] + 3)
        u1 = np.empty(n, dtype=np.float64)
        u2 = np.empty(n, dtype=np.float64)
        lib().orc_inlet_profile(self._h, u1.ctypes.data, u2.ctypes.data)
        return u1, u2

    def close(self) -> None:
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# the compiled reference harness (oracle/_ref)
# ---------------------------------------------------------------------------

def read_ref_dump(path: str, with_pops: bool = False) -> dict:
    """Parse the binary written by oracle/ref_harness.inc."""
    with open(path, "rb") as fh:
        hdr = np.frombuffer(fh.read(32), dtype=np.int32)
        inx, iny, nz, mnx, mny, ia, ib, steps = (int(v) for v in hdr)
        data = np.frombuffer(fh.read(), dtype=np.float64)
    n0 = inx * iny * nz
    n1 = mnx * mny * nz
    out = {"hdr": dict(inx=inx, iny=iny, nz=nz, mnx=mnx, mny=mny, ia=ia, ib=ib, steps=steps)}
    o = 0
    for box, n, shp in ((0, n0, (inx, iny, nz)), (1, n1, (mnx, mny, nz))):
        for name in FIELDS:
            out[(box, name)] = data[o:o + n].reshape(shp)
            o += n
    if with_pops:
        for box, n, shp in ((0, n0, (inx, iny, nz)), (1, n1, (mnx, mny, nz))):
            for fld in range(4):
                out[(box, "pops", fld)] = data[o:o + 19 * n].reshape((19,) + shp)
                o += 19 * n
    return out


def read_ref_mixing(path: str) -> np.ndarray:
    rows = []
    with open(path) as fh:
        for line in fh:
            parts = line.split()
            if len(parts) == 7 and parts[0].lstrip("-").isdigit():
                rows.append([float(x) for x in parts])
    return np.array(rows, dtype=np.float64)


def read_ref_pressure(path: str) -> dict:
    """The three zones of the reference's Pressure_<steps>.dat as arrays of
    rows {index, value, value * unit, third column}."""
    zones, cur = {}, None
    with open(path) as fh:
        for line in fh:
            if line.startswith("ZONE"):
                cur = line.split('"')[1]
                zones[cur] = []
                continue
            parts = line.split()
            if cur and len(parts) == 4:
                zones[cur].append([float(x) for x in parts])
    return {k: np.array(v, dtype=np.float64) for k, v in zones.items()}


def run_ref(binary: str, steps: int, with_pops: bool = False, threads: int | None = None, warmup: int = 0,
            writers: str | None = None):
    """Run a reference binary in a scratch directory; return (dump, mixing
    rows, seconds of the timed loop: the steps after the first ``warmup``).
    writers="domain" or "pvc" also collects the reference's Domain_Data (and
    Data_P_V_C) files as bytes in dump["files"]."""
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    with tempfile.TemporaryDirectory() as d:
        args = [binary, str(steps), os.path.join(d, "out.bin")] + (["pops"] if with_pops else [])
        if warmup:
            args.append("warmup=%d" % warmup)
        if writers:
            args.append("writers=%s" % writers)
        r = subprocess.run(args, cwd=d, env=env, capture_output=True, text=True, check=True)
        secs = None
        for line in r.stderr.splitlines():
            if line.startswith("TMXH_LOOP_SECONDS"):
                secs = float(line.split()[1])
        dump = read_ref_dump(os.path.join(d, "out.bin"), with_pops)
        mix = read_ref_mixing(os.path.join(d, "MixingQuality_%d.dat" % steps))
        dump["pressure"] = read_ref_pressure(os.path.join(d, "Pressure_%d.dat" % steps))
        dump["files"] = {}
        for name in ("Domain_Data_%d.dat" % steps, "Data_P_V_C%d.dat" % steps):
            if os.path.exists(os.path.join(d, name)):
                with open(os.path.join(d, name), "rb") as fh:
                    dump["files"][name.split("%d" % steps)[0].rstrip("_")] = fh.read()
    return dump, mix, secs
