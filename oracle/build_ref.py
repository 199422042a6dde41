"""Build recipe for the reference's own kernels (test infrastructure only).

Compiles, from the read-only reference tree into ``oracle/_ref/``
(git-ignored, shipped with the working tree so a machine without the
reference tree can still load it):

* the CPU PP kernel ``pp_force_kernel.c``, one library per layout;
* the CUDA path ``pp_force_kernel.cu`` + ``pm3_fft_cuda.cu`` for sm_100a, one
  library per layout (``build_gpu_one``).

The reference hard-codes its layout in file-scope constants
(pp_force_kernel.c:8-29: ng, nnt, nns, ratio_cs, ngb, ncore, nteam, nnest,
app).  For each layout listed in ``oracle/layouts.py`` the source is streamed
through a substitution of exactly those constant lines and fed to gcc on
stdin; no copy of the source is written anywhere.  ``ref_hooks.h`` is
force-included so that the internal arrays of c_pp_force_kernel_tile can be
captured for bit-exact binning checks (see ref_hooks.c).

The CUDA sources read their layout from a generated header
(``cuda_parameters_generated.h``, written by the reference's
tools/gen_cuda_parameters.py from parameters.f90).  Here that header is written
from the layout table instead, into the build's own directory under
``oracle/_ref/``; each source is streamed to nvcc on stdin with that directory
on the include path, so the reference tree is only read.  The nvcc flags are
the reference's (Makefile:74,77) with the architecture changed to sm_100a.

Usage:  python oracle/build_ref.py            (build every registered layout)
"""
from __future__ import annotations

import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from layouts import GPU_BUILDS, REF_BUILDS, ref_gpu_lib_name, ref_lib_name  # noqa: E402

REF_TREE = os.environ.get("CUBE_REFERENCE_DIR", "/root/reference")
REF_SRC = os.environ.get("CUBE_REFERENCE_SRC", os.path.join(REF_TREE, "pp_force_kernel.c"))
REF_CU_PP = os.path.join(REF_TREE, "pp_force_kernel.cu")
REF_CU_PM3 = os.path.join(REF_TREE, "pm3_fft_cuda.cu")
OUT_DIR = os.path.join(HERE, "_ref")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

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


def gpu_header(p: dict) -> str:
    """The reference's parameter header (cuda_parameters_generated.h:4-14) for layout p."""
    return "\n".join([
        "// written by oracle/build_ref.py for one layout of the reference's CUDA path",
        "#pragma once",
        f"constexpr int CUBE_NG = {int(p['ng'])};",
        f"constexpr int CUBE_NNT = {int(p['nnt'])};",
        f"constexpr int CUBE_NNS = {int(p['nns'])};",
        f"constexpr int CUBE_RATIO_CS = {int(p['ratio_cs'])};",
        f"constexpr int CUBE_NP_NC = {int(p['np_nc'])};",
        f"constexpr int CUBE_NGB = {int(p['ngb'])};",
        f"constexpr int CUBE_NCORE = {int(p['ncore'])};",
        "constexpr bool CUBE_BODY_CENTERED_CUBIC = false;",
        f"constexpr double CUBE_IMAGE_BUFFER = {float(p['image_buffer'])!r};",
        f"constexpr double CUBE_TILE_BUFFER = {float(p['tile_buffer'])!r};",
        f"constexpr double CUBE_APP = {float(p['app'])!r};",
        ""])


def build_gpu_one(p: dict, force: bool = False) -> str:
    """Compile the reference's CUDA PP + PM3 for layout p into one shared library."""
    os.makedirs(OUT_DIR, exist_ok=True)
    name = ref_gpu_lib_name(p)
    out = os.path.join(OUT_DIR, name)
    deps = [REF_CU_PP, REF_CU_PM3, __file__, os.path.join(HERE, "layouts.py")]
    if not force and os.path.exists(out):
        if all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps if os.path.exists(d)):
            return out
    inc = os.path.join(OUT_DIR, name[:-3] + ".inc")
    os.makedirs(inc, exist_ok=True)
    with open(os.path.join(inc, "cuda_parameters_generated.h"), "w") as f:
        f.write(gpu_header(p))
    objs = []
    # Makefile:74 (PP: -O3 -use_fast_math -DCUDA -fopenmp) and Makefile:77 (PM3: -O3)
    for src, extra in ((REF_CU_PP, ["-use_fast_math", "-DCUDA", "-Xcompiler", "-fopenmp,-fPIC"]),
                       (REF_CU_PM3, ["-Xcompiler", "-fPIC"])):
        obj = os.path.join(inc, os.path.basename(src) + ".o")
        cmd = [NVCC, "-x", "cu", "-", "-I", inc, "-O3", *ARCH, "-diag-suppress", "177,550", *extra,
               "-c", "-o", obj]
        with open(src, "rb") as f:
            subprocess.run(cmd, input=f.read(), check=True)
        objs.append(obj)
    subprocess.run([NVCC, *ARCH, "-shared", *objs, "-o", out, "-lcufft", f"-L{CUDA_HOME}/lib64",
                    f"-Xlinker=-rpath,{CUDA_HOME}/lib64", "-Xcompiler", "-fopenmp", "-Xlinker", "-Bsymbolic"],
                   check=True)
    for o in objs:
        os.remove(o)
    return out


def build_gpu_all(force: bool = False) -> list[str]:
    if not (os.path.exists(REF_CU_PP) and os.path.exists(REF_CU_PM3)):
        raise FileNotFoundError(REF_CU_PM3)
    return [build_gpu_one(p, force) for p in GPU_BUILDS.values()]


def build_all(force: bool = False) -> list[str]:
    if not os.path.exists(REF_SRC):
        raise FileNotFoundError(REF_SRC)
    return [build_one(p, force) for p in REF_BUILDS] + build_gpu_all(force)


if __name__ == "__main__":
    for path in build_all(force="--force" in sys.argv):
        print(path)
