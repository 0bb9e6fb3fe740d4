"""Generate the golden fixtures in tests/golden/ by running the reference
itself (Tmixer.cpp compiled by oracle/build_ref.py) on small cases.

Each fixture ``<name>.npz`` holds, after ``steps`` full steps of the
reference: the seven macroscopic fields of both boxes (``b0_rho`` ...
``b1_cC``), the mixing-quality rows the reference prints (17 significant
digits), and the case as JSON (``case``).

``reference_case_100.json`` pins the reference's own hard-coded case
(401x51x51 + 101x750x51, 4.9M nodes) after 100 steps by SHA-256 digests of
the little-endian FP64 bytes of each field of each box in [i][j][k] order and
of the mixing rows (the fields themselves would be 275 MB).  It needs about
10 GB of memory and a minute on 8 cores.

Needs /root/reference; run from the repository root:
    python tests/golden/make_golden.py [--full]
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


def full_reference_case() -> None:
    binary = build_ref.build("golden_reference_case", {})  # the reference's own constants
    dump, mix, secs = oracle.run_ref(binary, FULL_STEPS, threads=os.cpu_count())
    out = {"steps": FULL_STEPS, "fields": {"b%d_%s" % (b, f): digest(dump[(b, f)]) for b in (0, 1)
                                            for f in oracle.FIELDS},
           "mixing": digest(mix), "mixing_rows": int(mix.shape[0])}
    path = os.path.join(HERE, "reference_case_%d.json" % FULL_STEPS)
    with open(path, "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", path, "(reference loop %.1f s)" % secs)


def main() -> int:
    if "--full" in sys.argv:
        full_reference_case()
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
