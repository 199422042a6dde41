"""Layouts for which the reference's kernels are prebuilt (test infrastructure).

Each entry fixes the compile-time constants of the reference's
pp_force_kernel.c:8-29.  ``ngb`` is the tile buffer in fine cells
(ncb = ngb / ratio_cs coarse cells).  The fine-scale kick needs a one
coarse-cell buffer, so the workloads here use ngb = ratio_cs (ncb = 1); one
small layout keeps ncb = 2 to cover buffers deeper than the PP halo.

``GPU_BUILDS`` lists the builds of the reference's CUDA path
(pp_force_kernel.cu + pm3_fft_cuda.cu) for sm_100a.  Each fixes the eleven
constants of the reference's generated parameter header
(cuda_parameters_generated.h:4-14).  ``image_buffer`` and ``tile_buffer`` size
the reference's capacities np_image_max and np_tile_max
(pp_force_kernel.cu:45-51); clustered images need more than the reference's
defaults (2 and 3), which are parameters of its own parameters.f90.
"""
from __future__ import annotations

# name -> layout constants (app is the PP softening in fine cells)
LAYOUTS = {
    # small multi-tile layout used by most parity tests: nc=8, nt=4, ntt=2
    "t32": dict(ng=32, nnt=2, nns=2, ratio_cs=4, ngb=4, app=0.1),
    # single tile with a two coarse-cell buffer: nc=8, nt=8, ntt=4, ncb=2
    "t32b": dict(ng=32, nnt=1, nns=2, ratio_cs=4, ngb=8, app=0.1),
    # one periodic 64^3 box (Zel'dovich lattice workload), nt=16, ntt=8
    "cfg0": dict(ng=64, nnt=1, nns=2, ratio_cs=4, ngb=4, app=0.1),
    # a 96^3 clustered box as 2^3 tiles: nt=12, ntt=6
    "c96": dict(ng=96, nnt=2, nns=2, ratio_cs=4, ngb=4, app=0.1),
    # 256^3 clustered box as 2^3 tiles, nt=32, ntt=16
    "cfg1": dict(ng=256, nnt=2, nns=2, ratio_cs=4, ngb=4, app=0.1),
    # one tile of 256 coarse cells: float keys round across coarse cells for c >= 128
    "spill": dict(ng=1024, nnt=1, nns=1, ratio_cs=4, ngb=4, app=0.1),
}

# thread counts of the reference's nested OpenMP loops (pp_force_kernel.c:19-21)
_NNEST_TEST = 8
_NNEST_BENCH = (8, 16, 32, 64, 128, 256)


def _ref_params(layout: dict, nnest: int, nteam: int = 1) -> dict:
    p = dict(layout)
    p.update(ncore=nteam * nnest, nteam=nteam, nnest=nnest)
    return p


REF_BUILDS = [_ref_params(LAYOUTS[n], _NNEST_TEST) for n in ("t32", "t32b", "cfg0", "c96", "spill")]
REF_BUILDS += [_ref_params(LAYOUTS["cfg1"], k) for k in _NNEST_BENCH]
REF_BUILDS += [_ref_params(LAYOUTS["cfg0"], k) for k in _NNEST_BENCH if k != _NNEST_TEST]


def ref_lib_name(p: dict) -> str:
    app = ("%g" % p["app"]).replace(".", "p")
    return (f"libppref_ng{p['ng']}_nnt{p['nnt']}_nns{p['nns']}_cs{p['ratio_cs']}_ngb{p['ngb']}"
            f"_app{app}_team{p['nteam']}_nest{p['nnest']}.so")


def _gpu_params(layout: dict, **over) -> dict:
    p = dict(layout)
    p.update(np_nc=layout["ratio_cs"], ncore=16, image_buffer=4.0, tile_buffer=8.0)
    p.update(over)
    return p


# name -> constants of one build of the reference's CUDA path
GPU_BUILDS = {
    "t32": _gpu_params(LAYOUTS["t32"]),
    "t32b": _gpu_params(LAYOUTS["t32b"]),
    "cfg0": _gpu_params(LAYOUTS["cfg0"]),
    "c96": _gpu_params(LAYOUTS["c96"]),
    # the bench's clustered256 image (2^3 tiles of 32^3 coarse cells): parity and timing at scale
    "cfg1": _gpu_params(LAYOUTS["cfg1"]),
    # t32's image with one subtile per tile: the reference PM3 then solves one mesh of
    # (nt + 2) ratio_cs points per tile, the geometry of PM2 when ngb = ratio_cs
    "t32s1": _gpu_params(dict(LAYOUTS["t32"], nns=1)),
}


def ref_gpu_lib_name(p: dict) -> str:
    app = ("%g" % p["app"]).replace(".", "p")
    ib = ("%g" % p["image_buffer"]).replace(".", "p")
    tb = ("%g" % p["tile_buffer"]).replace(".", "p")
    return (f"libcuref_ng{p['ng']}_nnt{p['nnt']}_nns{p['nns']}_cs{p['ratio_cs']}_ngb{p['ngb']}"
            f"_app{app}_ib{ib}_tb{tb}_core{p['ncore']}.so")
