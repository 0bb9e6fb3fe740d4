"""tmixer_b200 -- B200-native coupled D3Q19 lattice-Boltzmann T-mixer solver.

Host-side mirror of the reference's driver (Tmixer.cpp:10413-10490) over the
C ABI of ``libtmx.so`` (``include/tmx.h``).  The reference is a single program
whose interface is its case ``#define`` block and five phase functions; here a
``CaseSpec`` carries the case and a ``Solver`` runs it on one GPU:

    spec = tmixer_b200.reference_case()          # Tmixer.cpp:76-149
    with tmixer_b200.Solver(spec) as s:           # allocateMemory()
        s.init()                                  # inlet profile + initial state
        s.step(1000)                              # 1000 x {eq, collide, stream, BC, moments}
        rho = s.field(0, "rho")                   # inlet-box density, shape (inx, iny, nz)
        rows, im = s.mixing()                     # write_MixingQuality numbers

There is no CPU fallback: every call goes to the CUDA library, and importing
the package fails loudly if ``libtmx.so`` is missing.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
from typing import Optional, Sequence

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libtmx.so")

FIELDS = ("rho", "ux", "uy", "uz", "cA", "cB", "cC")
TMX_FP64 = 0  # plain form, bit-exact with the reference
TMX_FP32 = 1  # FP32 storage and arithmetic
TMX_FP16 = 2  # FP32 arithmetic, populations stored in FP16 as f_q - feq_q of the writing node
PRECISIONS = {"fp64": TMX_FP64, "fp32": TMX_FP32, "fp16": TMX_FP16}
ABI_VERSION = 1

_ERRORS = {-1: "invalid", -2: "out of memory", -3: "CUDA error", -4: "bad call order", -5: "non-finite state"}


class TmxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("tmx error %d (%s): %s" % (code, _ERRORS.get(code, "?"), msg))
        self.code = code


class _CCase(ctypes.Structure):
    _fields_ = [("inx", ctypes.c_int), ("iny", ctypes.c_int), ("nz", ctypes.c_int),
                ("mnx", ctypes.c_int), ("mny", ctypes.c_int), ("ia", ctypes.c_int),
                ("tau", ctypes.c_double), ("tau_a", ctypes.c_double), ("tau_b", ctypes.c_double),
                ("tau_c", ctypes.c_double), ("rho0", ctypes.c_double), ("rho_out", ctypes.c_double),
                ("c_in", (ctypes.c_double * 2) * 3), ("rateconst", ctypes.c_double),
                ("umean", ctypes.c_double), ("precision", ctypes.c_int)]


class _CRequest(ctypes.Structure):
    _fields_ = [("c", _CCase), ("arrival", ctypes.c_double), ("max_steps", ctypes.c_int), ("window", ctypes.c_int),
                ("tol", ctypes.c_double)]


class _CServed(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("slot", ctypes.c_int), ("steps", ctypes.c_longlong),
                ("admitted", ctypes.c_double), ("finished", ctypes.c_double), ("outlet_im", ctypes.c_double * 3)]


class _CServeOpts(ctypes.Structure):
    _fields_ = [("check_every", ctypes.c_int), ("max_active", ctypes.c_int)]


_FOOTPRINT = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(_CCase), ctypes.POINTER(ctypes.c_longlong))
_CAPACITY = ctypes.CFUNCTYPE(ctypes.c_longlong, ctypes.c_void_p)
_ADD = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(_CCase), ctypes.POINTER(ctypes.c_int))
_REMOVE = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int)
_STEP = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int)
_OUTLET = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                           ctypes.POINTER(ctypes.c_double))
_NOW = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.c_void_p)
_WAIT = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_double)
_HEALTH = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                           ctypes.POINTER(ctypes.c_int))


class _CServeOps(ctypes.Structure):
    _fields_ = [("ctx", ctypes.c_void_p), ("footprint", _FOOTPRINT), ("capacity", _CAPACITY), ("add", _ADD),
                ("remove", _REMOVE), ("step", _STEP), ("outlet_im", _OUTLET), ("now", _NOW), ("wait_until", _WAIT),
                ("health", _HEALTH)]


_lib = None


def lib() -> ctypes.CDLL:
    """Load ``libtmx.so`` (built by ``tmixer_b200.build``); raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("tmixer_b200: %s is missing; run `python -m tmixer_b200.build`" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    L.tmx_abi_version.restype = ip
    L.tmx_last_error.restype = ctypes.c_char_p
    L.tmx_case_reference.argtypes = [P(_CCase)]
    L.tmx_case_check.argtypes = [P(_CCase)]
    L.tmx_case_footprint.argtypes = [P(_CCase), P(ctypes.c_longlong)]
    L.tmx_case_wlayout.argtypes = [ip, dp, dp, dp, dp, dp, P(_CCase)]
    L.tmx_create.argtypes = [P(_CCase), ip, P(vp)]
    L.tmx_init.argtypes = [vp]
    L.tmx_step.argtypes = [vp, ip]
    L.tmx_sync.argtypes = [vp]
    L.tmx_steps_done.argtypes = [vp]
    L.tmx_steps_done.restype = ctypes.c_longlong
    L.tmx_fields.argtypes = [vp, ip, ip, vp]
    L.tmx_populations.argtypes = [vp, ip, ip, vp]
    L.tmx_mixing.argtypes = [vp, vp, vp]
    L.tmx_mixing_static.argtypes = [vp, vp, vp]
    L.tmx_sums.argtypes = [vp, vp]
    L.tmx_pressure_power.argtypes = [vp, vp, vp, vp, vp]
    L.tmx_write_file.argtypes = [vp, ip, ctypes.c_char_p]
    L.tmx_case_of.argtypes = [vp, P(_CCase)]
    L.tmx_checkpoint_size.argtypes = [vp, P(ctypes.c_longlong)]
    L.tmx_checkpoint.argtypes = [vp, vp, ctypes.c_longlong]
    L.tmx_restore.argtypes = [vp, vp, ctypes.c_longlong]
    L.tmx_inlet_profile.argtypes = [vp, vp, vp]
    L.tmx_step_timed.argtypes = [vp, ip, P(dp), P(dp), P(dp)]
    L.tmx_counts.argtypes = [vp, P(ctypes.c_longlong)]
    L.tmx_set_shape.argtypes = [vp, ip, ip]
    L.tmx_time_steps.argtypes = [vp, ip, P(dp)]
    L.tmx_pattern_ceiling.argtypes = [ip, ctypes.c_longlong, ip, ip, P(dp), P(ip)]
    L.tmx_destroy.argtypes = [vp]
    L.tmx_destroy.restype = None
    LL = ctypes.c_longlong
    L.tmx_batch_footprint.argtypes = [P(_CCase), P(LL)]
    L.tmx_batch_create.argtypes = [ip, LL, ip, P(vp)]
    L.tmx_batch_add.argtypes = [vp, P(_CCase), P(ip)]
    L.tmx_batch_remove.argtypes = [vp, ip]
    L.tmx_batch_step.argtypes = [vp, ip, ip]
    L.tmx_batch_sync.argtypes = [vp]
    L.tmx_batch_slots.argtypes = [vp, P(ip), ip, P(ip)]
    L.tmx_batch_slot_steps.argtypes = [vp, ip]
    L.tmx_batch_slot_steps.restype = LL
    L.tmx_batch_outlet_im.argtypes = [vp, P(ip), ip, vp]
    L.tmx_batch_fields.argtypes = [vp, ip, ip, ip, vp]
    L.tmx_batch_health.argtypes = [vp, P(ip), ip, P(ip)]
    L.tmx_batch_info.argtypes = [vp, P(LL)]
    L.tmx_batch_set_shape.argtypes = [vp, ip, ip]
    L.tmx_batch_tune.argtypes = [vp, ip, P(ip), P(ip), P(dp)]
    L.tmx_batch_time_steps.argtypes = [vp, ip, P(dp)]
    L.tmx_batch_set_sweep.argtypes = [vp, ip, ip]
    L.tmx_batch_shape.argtypes = [vp, P(ip)]
    L.tmx_batch_set_boundary.argtypes = [vp, ip, ip]
    L.tmx_batch_step_timed.argtypes = [vp, ip, P(dp), P(dp), P(dp)]
    L.tmx_batch_boundary.argtypes = [vp, P(ip), P(ip)]
    L.tmx_batch_checkpoint_size.argtypes = [vp, ip, P(LL)]
    L.tmx_batch_checkpoint.argtypes = [vp, ip, vp, LL]
    L.tmx_batch_restore.argtypes = [vp, P(_CCase), vp, LL, P(ip)]
    L.tmx_batch_destroy.argtypes = [vp]
    L.tmx_batch_destroy.restype = None
    L.tmx_serve.argtypes = [vp, P(_CRequest), ip, P(_CServeOpts), P(_CServed), P(dp)]
    L.tmx_serve_with.argtypes = [P(_CServeOps), P(_CRequest), ip, P(_CServeOpts), P(_CServed), P(dp)]
    if L.tmx_abi_version() != ABI_VERSION:
        raise RuntimeError("libtmx.so ABI %d, expected %d" % (L.tmx_abi_version(), ABI_VERSION))
    _lib = L
    return L


def _check(rc: int) -> None:
    if rc != 0:
        raise TmxError(rc, lib().tmx_last_error().decode(errors="replace"))


@dataclasses.dataclass
class CaseSpec:
    """The reference's case constants (Tmixer.cpp:76-149) as runtime values.

    ``ia`` is the first inlet column over the opening; the last is
    ``ib = ia + mnx - 1`` (Tmixer.cpp:1374-1375).  ``c_in[s][n]`` is species s
    (A, B, C) at inlet n (1, 2).
    """
    inx: int
    iny: int
    nz: int
    mnx: int
    mny: int
    ia: int
    tau: float
    tau_a: float
    tau_b: float
    tau_c: float
    rho0: float
    rho_out: float
    c_in: Sequence[Sequence[float]]
    rateconst: float
    umean: float
    precision: int = TMX_FP64
    steps: int = 0  # the case's step count (the reference loops time+1 = 100001 times)

    @property
    def ib(self) -> int:
        return self.ia + self.mnx - 1

    def nodes(self) -> int:
        return self.inx * self.iny * self.nz + self.mnx * self.mny * self.nz

    def to_c(self) -> _CCase:
        c = _CCase()
        for k in ("inx", "iny", "nz", "mnx", "mny", "ia", "precision"):
            setattr(c, k, int(getattr(self, k)))
        for k in ("tau", "tau_a", "tau_b", "tau_c", "rho0", "rho_out", "rateconst", "umean"):
            setattr(c, k, float(getattr(self, k)))
        for s in range(3):
            for n in range(2):
                c.c_in[s][n] = float(self.c_in[s][n])
        return c

    @classmethod
    def from_c(cls, c: _CCase, steps: int = 0) -> "CaseSpec":
        return cls(inx=c.inx, iny=c.iny, nz=c.nz, mnx=c.mnx, mny=c.mny, ia=c.ia, tau=c.tau, tau_a=c.tau_a,
                   tau_b=c.tau_b, tau_c=c.tau_c, rho0=c.rho0, rho_out=c.rho_out,
                   c_in=[[c.c_in[s][n] for n in range(2)] for s in range(3)], rateconst=c.rateconst,
                   umean=c.umean, precision=c.precision, steps=steps)

    def as_dict(self) -> dict:
        """Plain-dict form (the oracle's parameter names)."""
        return dict(inx=self.inx, iny=self.iny, nz=self.nz, mnx=self.mnx, mny=self.mny, ia=self.ia,
                    tau=self.tau, taua=self.tau_a, taub=self.tau_b, taup=self.tau_c, rho0=self.rho0,
                    rho_out=self.rho_out, c0=0.0, cin=[list(r) for r in self.c_in],
                    rateconst=self.rateconst, umean=self.umean)

    def check(self) -> None:
        _check(lib().tmx_case_check(ctypes.byref(self.to_c())))

    def footprint(self) -> int:
        b = ctypes.c_longlong()
        _check(lib().tmx_case_footprint(ctypes.byref(self.to_c()), ctypes.byref(b)))
        return int(b.value)


def reference_case() -> CaseSpec:
    """The reference's hard-coded case: 401x51x51 inlet box, 101x750x51 mixing
    box, tau 0.6, Sc 3, Umean 0.059761, k 1.0, rho 3.0, 100001 steps."""
    c = _CCase()
    _check(lib().tmx_case_reference(ctypes.byref(c)))
    return CaseSpec.from_c(c, steps=100001)


def pattern_ceiling(precision: int, nodes: int, reps: int = 20, device: int = 0) -> dict:
    """The memory-traffic ceiling of the interior kernels' access pattern for
    one form (tmx_pattern_ceiling): GB/s of the form's bytes per lattice
    update, moved in its layout with no arithmetic, over at least ``nodes``
    nodes; the best of 1, 2, 4 and 8 blocks per SM."""
    g, b = ctypes.c_double(), ctypes.c_int()
    _check(lib().tmx_pattern_ceiling(int(precision), int(nodes), int(reps), int(device), ctypes.byref(g),
                                     ctypes.byref(b)))
    return dict(gbs=g.value, blocks_per_sm=b.value, nodes=int(nodes), reps=int(reps))

def w_layout(W: int, u_max: float, tau_f: float, tau_c: float, k: float, rho: float = 1.0,
             steps: int = 0, precision: int = TMX_FP64) -> CaseSpec:
    """A T-mixer of width W in the layout of the benchmark configurations:
    inlet 8W x W x W, mixing 2W x 4W x W, opening x = 3W+1 .. 5W, species A
    at inlet 1 and B at inlet 2 with c = 1, rho0 = rho_out = rho.  The duct
    profile is scaled so that its maximum is u_max (instead of the reference's
    mean Umean): umean is set to u_max * mean/max of the unscaled profile."""
    c = _CCase()
    _check(lib().tmx_case_wlayout(int(W), float(u_max), float(tau_f), float(tau_c), float(k), float(rho),
                                  ctypes.byref(c)))
    spec = CaseSpec.from_c(c, steps=steps)
    spec.precision = int(precision)
    return spec


class Solver:
    """One solve on one GPU: the device state of a ``CaseSpec``."""

    def __init__(self, spec: CaseSpec, device: int = 0):
        self.spec = spec
        self._h = ctypes.c_void_p()
        self._c = spec.to_c()
        _check(lib().tmx_create(ctypes.byref(self._c), int(device), ctypes.byref(self._h)))

    # -- lifecycle ---------------------------------------------------------
    def init(self) -> "Solver":
        _check(lib().tmx_init(self._h))
        return self

    def step(self, n: int = 1) -> "Solver":
        _check(lib().tmx_step(self._h, int(n)))
        return self

    def sync(self) -> None:
        _check(lib().tmx_sync(self._h))

    @property
    def steps_done(self) -> int:
        return int(lib().tmx_steps_done(self._h))

    def close(self) -> None:
        if self._h:
            lib().tmx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- outputs -------------------------------------------------------------
    def box_shape(self, box: int):
        s = self.spec
        return (s.inx, s.iny, s.nz) if box == 0 else (s.mnx, s.mny, s.nz)

    def field(self, box: int, name: str, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.box_shape(box), dtype=np.float64)
        assert out.dtype == np.float64 and out.flags.c_contiguous and out.shape == self.box_shape(box)
        _check(lib().tmx_fields(self._h, int(box), FIELDS.index(name), out.ctypes.data))
        return out

    def populations(self, box: int, fld: int) -> np.ndarray:
        out = np.empty((19,) + self.box_shape(box), dtype=np.float64)
        _check(lib().tmx_populations(self._h, int(box), int(fld), out.ctypes.data))
        return out

    def mixing(self):
        rows = np.empty((self.spec.mny + self.spec.iny, 7), dtype=np.float64)
        im = np.empty(3, dtype=np.float64)
        _check(lib().tmx_mixing(self._h, rows.ctypes.data, im.ctypes.data))
        return rows, im

    def mixing_static(self):
        """tmx_mixing_static: the rows of mixing() with no allocation inside
        the library call (fixed static device scratch, at most 4096 rows)."""
        rows = np.empty((self.spec.mny + self.spec.iny, 7), dtype=np.float64)
        im = np.empty(3, dtype=np.float64)
        _check(lib().tmx_mixing_static(self._h, rows.ctypes.data, im.ctypes.data))
        return rows, im

    def pressure_power(self):
        """(pressure rows (mny+iny, 3) {row, p, p - p_top}, inlet
        cross-sections (inx, 2) {i, p}, power rows (mny-2, 5) {j, section rate,
        total rate (both as the reference), the same summed over every x},
        units (P0, Pw0)) as tmx_pressure_power."""
        s = self.spec
        prow = np.empty((s.mny + s.iny, 3))
        px = np.empty((s.inx, 2))
        pw = np.empty((s.mny - 2, 5))
        units = np.empty(2)
        _check(lib().tmx_pressure_power(self._h, prow.ctypes.data, px.ctypes.data, pw.ctypes.data, units.ctypes.data))
        return prow, px, pw, units

    def checkpoint(self) -> bytes:
        """The solve's state (tmx_checkpoint) as bytes."""
        n = ctypes.c_longlong()
        _check(lib().tmx_checkpoint_size(self._h, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        _check(lib().tmx_checkpoint(self._h, buf, n.value))
        return buf.raw

    def restore(self, data: bytes) -> "Solver":
        """Replace the state with a checkpoint of the same case and form."""
        buf = ctypes.create_string_buffer(bytes(data), len(data))
        _check(lib().tmx_restore(self._h, buf, len(data)))
        return self

    FILE_KINDS = {"domain": 0, "pvc": 1, "pressure": 2, "mixing": 3}

    def write_file(self, kind: str, path: str) -> None:
        """One of the reference's Tecplot files ("domain" = Domain_Data,
        "pvc" = Data_P_V_C, "pressure", "mixing") from the last step."""
        _check(lib().tmx_write_file(self._h, self.FILE_KINDS[kind], os.fsencode(path)))

    def sums(self) -> np.ndarray:
        out = np.empty(8, dtype=np.float64)
        _check(lib().tmx_sums(self._h, out.ctypes.data))
        return out

    def inlet_profile(self):
        n = (self.spec.iny + 3, self.spec.nz + 3)
        u1 = np.empty(n, dtype=np.float64)
        u2 = np.empty(n, dtype=np.float64)
        _check(lib().tmx_inlet_profile(self._h, u1.ctypes.data, u2.ctypes.data))
        return u1, u2

    def step_timed(self, n: int):
        """Run n steps with CUDA events around every launch; returns
        (ms in the bulk kernel, ms in the boundary kernel, ms for the loop)."""
        a, b, t = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(lib().tmx_step_timed(self._h, int(n), ctypes.byref(a), ctypes.byref(b), ctypes.byref(t)))
        return a.value, b.value, t.value

    def time_steps(self, n: int) -> float:
        """Run n steps (the ``step`` path) between CUDA events on the solver's
        stream; returns the device time in ms."""
        ms = ctypes.c_double()
        _check(lib().tmx_time_steps(self._h, int(n), ctypes.byref(ms)))
        return ms.value

    def set_shape(self, kind: int, zchunk: int = 8) -> "Solver":
        """Launch shape of the interior kernel (tmx_set_shape): SHAPE_FLAT, or
        for the FP16 form a sweep shape (SHAPE_SWEEP8, SHAPE_SWEEP4) with zchunk
        planes per tile.  Every shape gives the same bits.  Default: SHAPE_SWEEP4
        with 8 planes for the FP16 form, SHAPE_FLAT for the others."""
        _check(lib().tmx_set_shape(self._h, int(kind), int(zchunk)))
        return self

    def counts(self) -> dict:
        o = (ctypes.c_longlong * 4)()
        _check(lib().tmx_counts(self._h, o))
        return dict(nodes=o[0], interior=o[1], boundary=o[2], device_bytes=o[3])


class Batch:
    """Many mixers of one precision stepped together (tmx_batch_*): one
    launch per kernel kind per step over all of them, state carved from one
    device arena of ``budget`` bytes."""

    def __init__(self, precision: int = TMX_FP16, budget: int = 1 << 30, device: int = 0):
        self.precision = int(precision)
        self._b = ctypes.c_void_p()
        self.specs = {}
        _check(lib().tmx_batch_create(self.precision, ctypes.c_longlong(int(budget)), int(device),
                                      ctypes.byref(self._b)))

    @staticmethod
    def footprint(spec: CaseSpec) -> int:
        c = spec.to_c()
        n = ctypes.c_longlong()
        _check(lib().tmx_batch_footprint(ctypes.byref(c), ctypes.byref(n)))
        return int(n.value)

    def add(self, spec: CaseSpec) -> int:
        c = spec.to_c()
        slot = ctypes.c_int()
        _check(lib().tmx_batch_add(self._b, ctypes.byref(c), ctypes.byref(slot)))
        self.specs[slot.value] = spec
        return slot.value

    def remove(self, slot: int) -> None:
        _check(lib().tmx_batch_remove(self._b, int(slot)))
        self.specs.pop(int(slot), None)

    def checkpoint(self, slot: int) -> bytes:
        n = ctypes.c_longlong()
        _check(lib().tmx_batch_checkpoint_size(self._b, int(slot), ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        _check(lib().tmx_batch_checkpoint(self._b, int(slot), buf, n.value))
        return buf.raw

    def restore(self, spec: CaseSpec, data: bytes) -> int:
        """Admit a mixer from a checkpoint of ``spec``; returns its slot."""
        c = spec.to_c()
        buf = ctypes.create_string_buffer(bytes(data), len(data))
        slot = ctypes.c_int()
        _check(lib().tmx_batch_restore(self._b, ctypes.byref(c), buf, len(data), ctypes.byref(slot)))
        self.specs[slot.value] = spec
        return slot.value

    def step(self, n: int = 1, write_macro: bool = True) -> "Batch":
        _check(lib().tmx_batch_step(self._b, int(n), 1 if write_macro else 0))
        return self

    def sync(self) -> None:
        _check(lib().tmx_batch_sync(self._b))

    def slots(self) -> list:
        n = ctypes.c_int()
        _check(lib().tmx_batch_slots(self._b, None, 0, ctypes.byref(n)))
        arr = (ctypes.c_int * max(1, n.value))()
        _check(lib().tmx_batch_slots(self._b, arr, n.value, ctypes.byref(n)))
        return list(arr[:n.value])

    def slot_steps(self, slot: int) -> int:
        return int(lib().tmx_batch_slot_steps(self._b, int(slot)))

    def outlet_im(self, slots=None) -> np.ndarray:
        """(len(slots), 3) outlet I_A, I_B, I_C after the last step that
        wrote the macroscopic fields."""
        slots = self.slots() if slots is None else list(slots)
        out = np.empty((len(slots), 3), dtype=np.float64)
        arr = (ctypes.c_int * max(1, len(slots)))(*slots)
        _check(lib().tmx_batch_outlet_im(self._b, arr, len(slots), out.ctypes.data))
        return out

    def health(self, slots=None) -> list:
        """1 for every mixer whose last macroscopic fields hold a non-finite
        value, else 0 (tmx_batch_health)."""
        slots = self.slots() if slots is None else list(slots)
        arr = (ctypes.c_int * max(1, len(slots)))(*slots)
        bad = (ctypes.c_int * max(1, len(slots)))()
        _check(lib().tmx_batch_health(self._b, arr, len(slots), bad))
        return list(bad[:len(slots)])

    def field(self, slot: int, box: int, name: str) -> np.ndarray:
        s = self.specs[int(slot)]
        shape = (s.inx, s.iny, s.nz) if box == 0 else (s.mnx, s.mny, s.nz)
        out = np.empty(shape, dtype=np.float64)
        _check(lib().tmx_batch_fields(self._b, int(slot), int(box), FIELDS.index(name), out.ctypes.data))
        return out

    def info(self) -> dict:
        o = (ctypes.c_longlong * 8)()
        _check(lib().tmx_batch_info(self._b, o))
        return dict(mixers=o[0], nodes=o[1], arena_bytes=o[2], free_bytes=o[3], threads=o[4], cells=o[5],
                    steps=o[6], table_bytes=o[7])

    def set_shape(self, threads: int, cells: int) -> None:
        """The flat interior kernel with this block size and cell-block size."""
        _check(lib().tmx_batch_set_shape(self._b, int(threads), int(cells)))

    def set_sweep(self, kind: int, zchunk: int) -> None:
        """One of the FP16 form's sweep interior kernels (a SHAPE_SWEEP* kind)
        with zchunk planes per tile."""
        _check(lib().tmx_batch_set_sweep(self._b, int(kind), int(zchunk)))

    def set_boundary(self, blocks_per_sm: int, after: bool = False) -> None:
        """The boundary kernels' persistent grid in blocks per SM (0: as many
        as fit), and whether the interior kernel runs after them (else beside
        them; the FP64 form always after)."""
        _check(lib().tmx_batch_set_boundary(self._b, int(blocks_per_sm), 1 if after else 0))

    def shape(self) -> dict:
        o = (ctypes.c_int * 4)()
        _check(lib().tmx_batch_shape(self._b, o))
        bb, ba = ctypes.c_int(), ctypes.c_int()
        _check(lib().tmx_batch_boundary(self._b, ctypes.byref(bb), ctypes.byref(ba)))
        return dict(kernel=SHAPE_NAMES[o[0]], threads=o[1], cells=o[2], zchunk=o[3],
                    nodes_per_thread=(o[2] // o[1]) if o[0] == SHAPE_FLAT else o[3],
                    boundary_blocks_per_sm=bb.value, interior_after_boundary=bool(ba.value))

    def set_from(self, shape: dict) -> None:
        """Apply a shape() dictionary (e.g. the tuned shape of another batch)."""
        if shape["kernel"] == "flat":
            self.set_shape(shape["threads"], shape["cells"])
        else:
            self.set_sweep(SHAPE_KINDS[shape["kernel"]], shape["zchunk"])
        if "boundary_blocks_per_sm" in shape:
            self.set_boundary(shape["boundary_blocks_per_sm"], shape.get("interior_after_boundary", False))

    def tune(self, steps_per_trial: int = 20) -> dict:
        """Autotune the interior kernel's shape (tmx_batch_tune) and return it
        with its time per step."""
        t, c, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        _check(lib().tmx_batch_tune(self._b, int(steps_per_trial), ctypes.byref(t), ctypes.byref(c),
                                    ctypes.byref(ms)))
        return dict(self.shape(), ms_per_step=ms.value, steps_per_trial=int(steps_per_trial))

    def time_steps(self, n: int) -> float:
        ms = ctypes.c_double()
        _check(lib().tmx_batch_time_steps(self._b, int(n), ctypes.byref(ms)))
        return ms.value

    def step_timed(self, n: int):
        """(interior ms, boundary ms, total ms) of n steps with each kernel
        timed alone (tmx_batch_step_timed)."""
        a, b, t = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(lib().tmx_batch_step_timed(self._b, int(n), ctypes.byref(a), ctypes.byref(b), ctypes.byref(t)))
        return a.value, b.value, t.value

    def close(self) -> None:
        if self._b:
            lib().tmx_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclasses.dataclass
class Request:
    """One solve of the served form: a case, its arrival time (seconds after
    the loop starts) and its stopping rule."""
    spec: CaseSpec
    arrival: float = 0.0
    max_steps: int = 50000
    window: int = 500
    tol: float = 1e-6

    def to_c(self) -> _CRequest:
        return _CRequest(self.spec.to_c(), float(self.arrival), int(self.max_steps), int(self.window),
                         float(self.tol))


SHAPE_FLAT, SHAPE_SWEEP8, SHAPE_SWEEP4 = 0, 1, 2
SHAPE_NAMES = {SHAPE_FLAT: "flat", SHAPE_SWEEP8: "sweep8", SHAPE_SWEEP4: "sweep4"}
SHAPE_KINDS = {v: k for k, v in SHAPE_NAMES.items()}

SERVE_STATUS = {0: "converged", 1: "max_steps", -2: "too large for the budget", -5: "non-finite"}


def _serve_out(reqs, res, summ):
    results = [dict(status=SERVE_STATUS.get(r.status, r.status), slot=r.slot, steps=r.steps, arrival=q.arrival,
                    admitted=r.admitted, finished=r.finished, time_to_solution=r.finished - q.arrival,
                    outlet_im=list(r.outlet_im)) for q, r in zip(reqs, res)]
    summary = dict(makespan_s=summ[0], lattice_updates=summ[1], mlups=summ[2], p50_s=summ[3], p99_s=summ[4],
                   max_active=int(summ[5]), mean_active=summ[6], checks=int(summ[7]))
    return results, summary


def serve(batch: "Batch", requests, check_every: int = 100, max_active: int = 0):
    """Run the request loop (tmx_serve) over a batch; returns (per-request
    results, summary with makespan, aggregate MLUPS and p50/p99 time to
    solution)."""
    reqs = list(requests)
    arr = (_CRequest * max(1, len(reqs)))(*[q.to_c() for q in reqs])
    res = (_CServed * max(1, len(reqs)))()
    opts = _CServeOpts(int(check_every), int(max_active))
    summ = (ctypes.c_double * 8)()
    _check(lib().tmx_serve(batch._b, arr, len(reqs), ctypes.byref(opts), res, summ))
    return _serve_out(reqs, res[:len(reqs)], summ)


def serve_with(engine, requests, check_every: int = 100, max_active: int = 0):
    """Run the same request loop (tmx_serve_with) over a Python engine object
    with methods footprint(spec), capacity(), add(spec) -> slot, None when it
    does not fit now, or a negative TMX_E_* code when it cannot take the case
    at all, remove(slot), step(n), outlet_im(slots) -> (n, 3),
    now(), wait_until(t), and optionally health(slots) -> list of 0/1 (1: the
    mixer's state is non-finite).  For tests of the scheduler without a GPU."""
    reqs = list(requests)
    errors = []

    def guard(fn, fail=-3):
        def w(*a):
            try:
                return fn(*a)
            except Exception as e:  # pragma: no cover - surfaced below
                errors.append(e)
                return fail
        return w

    def fp(_, c, out):
        out[0] = int(engine.footprint(CaseSpec.from_c(c.contents)))
        return 0

    def add(_, c, slot):
        s = engine.add(CaseSpec.from_c(c.contents))
        if s is None:
            return -2
        if int(s) < 0:  # the engine refuses this case (a TMX_E_* code)
            return int(s)
        slot[0] = int(s)
        return 0

    def rem(_, slot):
        engine.remove(int(slot))
        return 0

    def step(_, n):
        engine.step(int(n))
        return 0

    def im(_, slots, n, out):
        v = np.asarray(engine.outlet_im([slots[i] for i in range(n)]), dtype=np.float64).reshape(n, 3)
        for i in range(n):
            for s in range(3):
                out[3 * i + s] = float(v[i, s])
        return 0

    def health(_, slots, n, bad):
        v = engine.health([slots[i] for i in range(n)])
        for i in range(n):
            bad[i] = int(v[i])
        return 0

    cbs = [_FOOTPRINT(guard(fp)), _CAPACITY(guard(lambda _: int(engine.capacity()), 0)), _ADD(guard(add)),
           _REMOVE(guard(rem)), _STEP(guard(step)), _OUTLET(guard(im)), _NOW(guard(lambda _: float(engine.now()), 0.0)),
           _WAIT(guard(lambda _, t: engine.wait_until(float(t)), None)),
           _HEALTH(guard(health)) if hasattr(engine, "health") else _HEALTH()]
    ops = _CServeOps(None, *cbs)
    arr = (_CRequest * max(1, len(reqs)))(*[q.to_c() for q in reqs])
    res = (_CServed * max(1, len(reqs)))()
    opts = _CServeOpts(int(check_every), int(max_active))
    summ = (ctypes.c_double * 8)()
    rc = lib().tmx_serve_with(ctypes.byref(ops), arr, len(reqs), ctypes.byref(opts), res, summ)
    if errors:
        raise errors[0]
    _check(rc)
    return _serve_out(reqs, res[:len(reqs)], summ)


__all__ = ["SHAPE_FLAT", "SHAPE_SWEEP8", "SHAPE_SWEEP4", "CaseSpec", "Solver", "Batch", "Request", "serve", "serve_with", "TmxError", "FIELDS", "TMX_FP64", "TMX_FP32", "TMX_FP16", "PRECISIONS",
           "reference_case", "w_layout", "lib"]
