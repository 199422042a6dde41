"""Build recipe for the sm_100a shared library ``cube2_b200/libcube2_b200.so``.

Each ``csrc/*.cu`` is compiled by nvcc for ``arch=compute_100a,code=sm_100a``
with line info, then linked with cuFFT into one C-ABI shared library that
sits next to this file (built in-tree, so it travels with the working tree).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcube2_b200.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr"]
SOURCES = ["binning.cu", "pp.cu", "pm3.cu", "ewald.cu", "probe.cu", "noalloc.cu", "mlp.cu", "drift.cu", "power.cu", "snapshot.cu", "sums.cu", "fallback.cu", "api.cu"]
HEADERS = ["common.cuh"]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS]
    hdrs.append(os.path.join(HERE, "..", "include", "cube2_b200.h"))
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s, *hdrs, __file__]):
            cmd = [NVCC, *ARCH, *FLAGS, "-c", s, "-o", o]
            if verbose:
                cmd.append("-Xptxas=-v")
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", *objs, "-o", LIB, "-lcufft", f"-L{CUDA_HOME}/lib64",
               f"-Xlinker=-rpath,{CUDA_HOME}/lib64"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
