"""Generate the golden fixtures in tests/golden/ by running the reference
itself (Tmixer.cpp compiled by oracle/build_ref.py) on small cases.

Each fixture ``<name>.npz`` holds, after ``steps`` full steps of the
reference: the seven macroscopic fields of both boxes (``b0_rho`` ...
``b1_cC``), the mixing-quality rows the reference prints (17 significant
digits), and the case as JSON (``case``).  Needs /root/reference; run from the
repository root:  python tests/golden/make_golden.py
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


def main() -> int:
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
