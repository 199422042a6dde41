"""Build recipe for the reference CPU PP kernel (test infrastructure only).

Compiles the reference's own ``pp_force_kernel.c`` from the read-only
reference tree into ``oracle/_ref/`` (git-ignored, shipped with the working
tree so a machine without the reference tree can still load it).

The reference hard-codes its layout in file-scope constants
(pp_force_kernel.c:8-29: ng, nnt, nns, ratio_cs, ngb, ncore, nteam, nnest,
app).  For each layout listed in ``oracle/layouts.py`` the source is streamed
through a substitution of exactly those constant lines and fed to gcc on
stdin; no copy of the source is written anywhere.  ``ref_hooks.h`` is
force-included so that the internal arrays of c_pp_force_kernel_tile can be
captured for bit-exact binning checks (see ref_hooks.c).

Usage:  python oracle/build_ref.py            (build every registered layout)
"""
from __future__ import annotations

import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from layouts import REF_BUILDS, ref_lib_name  # noqa: E402

REF_SRC = os.environ.get("CUBE_REFERENCE_SRC", "/root/reference/pp_force_kernel.c")
OUT_DIR = os.path.join(HERE, "_ref")

# pp_force_kernel.c:8-29 -- the constant definitions that carry the layout.
_CONST_PATTERNS = {
    "ng": r"^const int ng = \d+;$",
    "nnt": r"^const int nnt = \d+;$",
    "nns": r"^const int nns = \d+;$",
    "ratio_cs": r"^const int ratio_cs = \d+;$",
    "ngb": r"^const int ngb = \d+;$",
    "ncore": r"^const int ncore = \d+;$",
    "nteam": r"^const int nteam = \d+;$",
    "nnest": r"^const int nnest = \d+;$",
    "app": r"^const double app = [0-9.eE+-]+;$",
}


def specialise(src: str, params: dict) -> str:
    """Return the reference source with the layout constants replaced."""
    out = src
    for name, pat in _CONST_PATTERNS.items():
        val = params[name]
        typ = "double" if name == "app" else "int"
        repl = f"const {typ} {name} = {val!r};" if name == "app" else f"const int {name} = {int(val)};"
        out, n = re.subn(pat, repl, out, count=1, flags=re.M)
        if n != 1:
            raise RuntimeError(f"reference constant line for {name!r} not found exactly once")
    return out


def build_one(params: dict, force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    out = os.path.join(OUT_DIR, ref_lib_name(params))
    deps = [REF_SRC, os.path.join(HERE, "ref_hooks.c"), os.path.join(HERE, "ref_hooks.h"), __file__,
            os.path.join(HERE, "layouts.py")]
    if not force and os.path.exists(out):
        if all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps if os.path.exists(d)):
            return out
    with open(REF_SRC) as f:
        src = specialise(f.read(), params)
    hooks_o = out + ".hooks.o"
    subprocess.run(["gcc", "-O3", "-fPIC", "-c", os.path.join(HERE, "ref_hooks.c"), "-o", hooks_o],
                   check=True)
    cmd = ["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", "-include", os.path.join(HERE, "ref_hooks.h"),
           "-x", "c", "-", "-x", "none", hooks_o, "-o", out, "-lm", "-Wl,-Bsymbolic"]
    subprocess.run(cmd, input=src.encode(), check=True)
    os.remove(hooks_o)
    return out


def build_all(force: bool = False) -> list[str]:
    if not os.path.exists(REF_SRC):
        raise FileNotFoundError(REF_SRC)
    return [build_one(p, force) for p in REF_BUILDS]


if __name__ == "__main__":
    for path in build_all(force="--force" in sys.argv):
        print(path)
