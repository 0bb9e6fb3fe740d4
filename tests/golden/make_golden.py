"""Generate the golden fixtures in tests/golden/ by running the reference
itself (Tmixer.cpp compiled by oracle/build_ref.py) on small cases.

Each fixture ``<name>.npz`` holds, after ``steps`` full steps of the
reference: the seven macroscopic fields of both boxes (``b0_rho`` ...
``b1_cC``), the mixing-quality rows the reference prints (17 significant
digits), and the case as JSON (``case``).

``reference_case_<STEPS>.json`` (``--full [STEPS]``, default 100) pins the
reference's own hard-coded case (401x51x51 + 101x750x51, 4.9M nodes) after
STEPS steps by SHA-256 digests of the little-endian FP64 bytes of each field
of each box in [i][j][k] order and of the mixing rows (the fields themselves
would be 275 MB).  It needs about 10 GB of memory; 100 steps take about three
minutes on 8 cores, 1,000 steps about half an hour.

``w32_<STEPS>.json`` (``--w32 [STEPS]``, default 20000) pins the single-mixer
benchmark case the same way: the W=32 T-mixer (inlet 256x32x32 + mixing
64x128x32, profile maximum 0.05, tau_f 0.6, tau_c 0.6, k 1e-3, rho 1; case
constants from bench.w_layout_params) after its full 20,000 steps, about
40 minutes on 8 cores.

Needs the reference source (oracle/build_ref.py: TMX_REF_SRC); run from the
repository root:
    python tests/golden/make_golden.py [--full [STEPS]] [--w32 [STEPS]]
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import build_ref, oracle  # noqa: E402
from tests.cases import GOLDEN_CASES, ref_params  # noqa: E402


FULL_STEPS = 100


def digest(a: np.ndarray) -> str:
    """SHA-256 of the FP64 bytes with -0 taken as +0 and every NaN as one
    quiet NaN (the comparisons elsewhere treat those as equal too)."""
    import hashlib

    a = np.asarray(a, dtype=np.float64) + 0.0
    a = np.where(np.isnan(a), np.float64("nan"), a)
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


W32_STEPS = 20000
W32_CASE = dict(W=32, u_max=0.05, tau_f=0.6, tau_c=0.6, k=1e-3, rho=1.0)


def digest_run(name: str, params: dict, steps: int, out_name: str, extra: dict | None = None) -> None:
    """Run the reference for ``steps`` steps and write the digests of its
    fields and mixing rows to tests/golden/<out_name>."""
    binary = build_ref.build(name, params)
    threads = int(os.environ.get("TMX_GOLDEN_THREADS", os.cpu_count() or 1))
    dump, mix, secs = oracle.run_ref(binary, steps, threads=threads)
    out = {"steps": steps, "fields": {"b%d_%s" % (b, f): digest(dump[(b, f)]) for b in (0, 1)
                                      for f in oracle.FIELDS},
           "mixing": digest(mix), "mixing_rows": int(mix.shape[0])}
    if extra:
        out.update(extra)
    path = os.path.join(HERE, out_name)
    with open(path, "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", path, "(reference loop %.1f s)" % secs)


def full_reference_case(steps: int = FULL_STEPS) -> None:
    # the reference's own constants
    digest_run("golden_reference_case", {}, steps, "reference_case_%d.json" % steps)


def w32_case(steps: int = W32_STEPS) -> None:
    import bench

    c = W32_CASE
    params = bench.w_layout_params(c["W"], c["u_max"], c["tau_f"], c["tau_c"], c["k"], c["rho"])
    digest_run("golden_w32", params, steps, "w32_%d.json" % steps, extra={"case": dict(c)})


def _steps_after(flag: str, default: int) -> int:
    i = sys.argv.index(flag)
    if i + 1 < len(sys.argv) and sys.argv[i + 1].isdigit():
        return int(sys.argv[i + 1])
    return default


def main() -> int:
    if "--full" in sys.argv or "--w32" in sys.argv:
        if "--w32" in sys.argv:
            w32_case(_steps_after("--w32", W32_STEPS))
        if "--full" in sys.argv:
            full_reference_case(_steps_after("--full", FULL_STEPS))
        return 0
    for name, (case, steps) in GOLDEN_CASES.items():
        binary = build_ref.build("golden_" + name, ref_params(case))
        dump, mix, _ = oracle.run_ref(binary, steps, threads=1)
        arrays = {"b%d_%s" % (b, f): dump[(b, f)] for b in (0, 1) for f in oracle.FIELDS}
        arrays["mixing"] = mix
        arrays["case"] = np.array(json.dumps(dict(case, steps=steps)))
        out = os.path.join(HERE, name + ".npz")
        np.savez_compressed(out, **arrays)
        print("wrote", out, os.path.getsize(out), "bytes")
    return 0


if __name__ == "__main__":
    sys.exit(main())
