"""Build recipe for ``oracle/_ref``: the reference solver compiled from its own
source, ``Tmixer.cpp``, for one case.  Test infrastructure only.

The reference fixes every case parameter with an unguarded ``#define``
(Tmixer.cpp:76-149), so ``-D`` cannot override them.  This script reads the
source where it lies, applies the substitutions below in memory, appends the
harness ``oracle/ref_harness.inc`` and pipes the result to ``g++ -x c++ -``.  No
copy of the reference source is written anywhere; the only output is the
binary under ``oracle/_ref/``.

Substitutions (each one a parameter of the case, not a change of algorithm):
  * the size, relaxation, inlet, reaction and density defines (Tmixer.cpp:84-149);
  * ``ib = ia + mnx - 1`` (Tmixer.cpp:1375): identical for the odd widths the
    reference uses, and the only form that opens ``mnx`` columns for even widths;
  * ``amax``/``bmax``/``sumy*`` start at 0 (Tmixer.cpp:10171-10175 read them
    uninitialised);
  * the mixing-quality and pressure/power rows print 17 significant digits
    instead of ``%g``
    (Tmixer.cpp:10300-10401);
  * the reference ``main`` (Tmixer.cpp:10413) is renamed so the harness drives
    the phase functions itself.

usage: python oracle/build_ref.py NAME key=value ...   (prints the binary path)
"""
from __future__ import annotations

import hashlib
import json
import os
import re
import subprocess
import sys

# The reference source: TMX_REF_SRC names it; the default is where the
# reference is mounted in the build container.
REF_SRC = os.environ.get("TMX_REF_SRC", "/root/reference/Tmixer.cpp")
HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
HARNESS = os.path.join(HERE, "ref_harness.inc")

# Reference case (Tmixer.cpp:84-149).  tau_c None keeps the reference's
# Schmidt-number formula for taua/taub/taup (Tmixer.cpp:86-88).
REFERENCE_CASE = dict(inx=401, iny=51, nz=51, mnx=101, mny=750, tau=0.6, tau_c=None,
                      umean=0.059761, rateconst=1.0, rho0=3.0, rho_out=3.0,
                      ca_in1=1.0, ca_in2=0.0, cb_in1=0.0, cb_in2=1.0,
                      cp_in1=0.0, cp_in2=0.0)


def _fmt(v: float) -> str:
    r = repr(float(v))
    return r if ("." in r or "e" in r or "inf" in r or "nan" in r) else r + ".0"


def patched_source(params: dict) -> str:
    p = dict(REFERENCE_CASE)
    p.update(params)
    with open(REF_SRC, "r", encoding="latin-1") as fh:
        src = fh.read()

    def define(name: str, value: str) -> None:
        nonlocal src
        pat = re.compile(r"^#define %s\b.*$" % re.escape(name), re.M)
        if len(pat.findall(src)) != 1:
            raise RuntimeError("expected one #define %s in the reference" % name)
        src = pat.sub("#define %s %s" % (name, value), src, count=1)

    for k in ("inx", "iny", "nz", "mnx", "mny"):
        define(k, "(%d)" % int(p[k]))
    define("tau", "(%s)" % _fmt(p["tau"]))
    if p.get("tau_c") is not None:
        for k in ("taua", "taub", "taup"):
            define(k, "(%s)" % _fmt(p["tau_c"]))
    define("Umean", "(%s)" % _fmt(p["umean"]))
    define("rateconst", "(%s)" % _fmt(p["rateconst"]))
    define("rho_out", "(%s)" % _fmt(p["rho_out"]))
    define("rho0", "(%s)" % _fmt(p["rho0"]))
    for k, name in (("ca_in1", "Ca_in1"), ("ca_in2", "Ca_in2"), ("cb_in1", "Cb_in1"),
                    ("cb_in2", "Cb_in2"), ("cp_in1", "Cp_in1"), ("cp_in2", "Cp_in2")):
        define(name, "(%s)" % _fmt(p[k]))

    def sub1(old: str, new: str) -> None:
        nonlocal src
        if src.count(old) != 1:
            raise RuntimeError("expected one occurrence of %r" % old)
        src = src.replace(old, new)

    sub1("int ib = ((inx + 1) / 2) + ((mnx - 1) / 2);", "int ib = ia + mnx - 1;")
    sub1("double amax,bmax,cmax;", "double amax = 0, bmax = 0, cmax = 0;")
    sub1("double sumx,  sumz,  sumy; ", "double sumx = 0, sumz = 0, sumy = 0; ")
    sub1("double sumx_b,sumz_b,sumy_b; ", "double sumx_b = 0, sumz_b = 0, sumy_b = 0; ")
    sub1("double sumx_c,sumz_c,sumy_c; ", "double sumx_c = 0, sumz_c = 0, sumy_c = 0; ")
    n = src.count('"%d\\t%g\\t%g\\t%g\\t%g\\t%g\\t%g\\n"')
    if n != 4:
        raise RuntimeError("expected 4 mixing-quality formats, found %d" % n)
    src = src.replace('"%d\\t%g\\t%g\\t%g\\t%g\\t%g\\t%g\\n"',
                      '"%d\\t%.17g\\t%.17g\\t%.17g\\t%.17g\\t%.17g\\t%.17g\\n"')
    n = src.count('"%d\\t%g\\t%g\\t%g\\n"')
    if n != 4:
        raise RuntimeError("expected 4 pressure/power formats, found %d" % n)
    src = src.replace('"%d\\t%g\\t%g\\t%g\\n"', '"%d\\t%.17g\\t%.17g\\t%.17g\\n"')
    sub1("int main()\n", "int tmx_reference_main_unused()\n")
    with open(HARNESS, "r") as fh:
        src += "\n" + fh.read()
    return src


def binary_path(name: str, params: dict) -> str:
    """Binary name: case parameters plus the harness and this recipe, so a
    changed harness or patch list never reuses a stale binary."""
    key = json.dumps({k: params[k] for k in sorted(params)}, sort_keys=True)
    with open(HARNESS, "rb") as fh:
        key += hashlib.sha1(fh.read()).hexdigest()
    with open(os.path.abspath(__file__), "rb") as fh:
        key += hashlib.sha1(fh.read()).hexdigest()
    h = hashlib.sha1(key.encode()).hexdigest()[:10]
    return os.path.join(OUT_DIR, "tmixer_ref_%s_%s" % (name, h))


def build(name: str, params: dict, force: bool = False) -> str:
    """Compile the reference for ``params`` (see REFERENCE_CASE) and return the
    binary path.  Requires the reference source; reuses an existing binary."""
    out = binary_path(name, params)
    if os.path.exists(out) and not force:
        return out
    os.makedirs(OUT_DIR, exist_ok=True)
    src = patched_source(params)
    tmp = out + ".tmp"
    cmd = ["g++", "-O2", "-fopenmp", "-w", "-x", "c++", "-", "-o", tmp, "-lm"]
    subprocess.run(cmd, input=src.encode("latin-1"), check=True)
    os.replace(tmp, out)
    return out


def main(argv: list[str]) -> int:
    if len(argv) < 2:
        print(__doc__)
        return 2
    name = argv[1]
    params = {}
    for kv in argv[2:]:
        k, v = kv.split("=", 1)
        params[k] = None if v == "None" else (int(v) if k in ("inx", "iny", "nz", "mnx", "mny") else float(v))
    print(build(name, params, force=True))
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
