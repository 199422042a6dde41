"""Named fine-scale-kick workloads (seeded synthetic inputs in the reference layout).

* ``zeldovich64``   64^3 particles on a 64^3-fine-cell periodic box: lattice
  displaced by the Zel'dovich field of a P(k) ~ k^-2 Gaussian field, rms
  displacement 0.5 cell (seed 1000).  PM3 mesh 128^3, PP cutoff 2 fine cells,
  softening 0.1 cell.  One tile (nnt = 1).
* ``clustered256``  Poisson sample (mean 1 per fine cell, ~16.8M particles)
  of a lognormal density on a 256^3 box, sigma_lnrho = 1.5, P(k) ~ k^-2
  (seed 2000); fine-cell occupancy 0 to several hundred.  PM3 mesh 512^3, PP
  cutoff 2 fine cells, softening 0.1.  2^3 tiles (nnt = 2).

* ``batch512``      512 independent periodic boxes of 32^3 fine cells stored as
  the 8^3 parent tiles of one image (PM3 geometry CUBE_PM3_TILE_PERIODIC: a
  64^3 mesh per box).  Box t holds an m^3 lattice displaced by its own
  Zel'dovich field (seed 3000 + t, rms 0.5 cell), m^3 the nearest cube to a
  lognormal count (median 32^3, sigma 1, clipped to 2048 .. 200000; seed
  3000), so the boxes are uneven.  ``batch8`` is the same with 8 boxes.

* ``loop512``       the kick-drift time loop: 512^3 particles on a 512^3-fine-cell box
  (PM3 mesh 1024^3), Zel'dovich initial conditions (P(k) ~ k^-2, rms displacement 0.5
  cell, seed 5000) built on the device (cube2_b200/loop.py), 2^3 tiles.  ``loop128``
  and ``loop256`` are the same at 128^3 (tests and quick runs) and 256^3 (profiling).

All use ratio_cs = 4, a one coarse-cell tile buffer (ngb = 4), TSC, equal
particle mass 1, PM3 softening apm3f = 4 mesh cells on a ratio_sf = 2 mesh
(so the PP range apm3f / ratio_sf is 2 fine cells) and the full periodic
force (apm_range = 0).
"""
from __future__ import annotations

import os

import numpy as np

from . import ic
from .layout import RATIO_SF, Image, Layout, apm3_table, build_image, build_tile_batch, ixyz3_table

WORKLOADS = {
    "zeldovich64": dict(layout=dict(ng=64, nnt=1, nns=2, ratio_cs=4, ngb=4, app=0.1), kind="zeldovich", n=64,
                        rms=0.5, seed=1000, rsf=2, apm3f=4.0),
    "clustered256": dict(layout=dict(ng=256, nnt=2, nns=2, ratio_cs=4, ngb=4, app=0.1), kind="lognormal", n=256,
                         sigma=1.5, seed=2000, rsf=2, apm3f=4.0),
    # profiling size: same statistics, 192^3 box (~7M particles), 384^3 mesh (> L2 per array)
    "clustered192": dict(layout=dict(ng=192, nnt=2, nns=2, ratio_cs=4, ngb=4, app=0.1), kind="lognormal", n=192,
                         sigma=1.5, seed=2000, rsf=2, apm3f=4.0),
    # 512 independent periodic boxes of 32^3 fine cells, uneven particle counts, one launch per stage
    "batch512": dict(layout=dict(ng=256, nnt=8, nns=2, ratio_cs=4, ngb=4, app=0.1), kind="batch", box=32,
                     median=32768, sigma=1.0, clip=(2048, 200000), seed=3000, rsf=2, apm3f=4.0),
    # the same with 8 boxes and smaller counts (tests)
    "batch8": dict(layout=dict(ng=64, nnt=2, nns=2, ratio_cs=4, ngb=4, app=0.1), kind="batch", box=32,
                   median=4096, sigma=1.0, clip=(512, 20000), seed=3100, rsf=2, apm3f=4.0),
}

# time loops: initial conditions built on the device (loop.zeldovich_start)
LOOP_WORKLOADS = {
    "loop512": dict(layout=dict(ng=512, nnt=2, nns=2, ratio_cs=4, ngb=4, app=0.1), rms=0.5, seed=5000, apm3f=4.0,
                    growth_per_step=0.05, pk_grid=512),
    "loop128": dict(layout=dict(ng=128, nnt=2, nns=2, ratio_cs=4, ngb=4, app=0.1), rms=0.5, seed=5100, apm3f=4.0,
                    growth_per_step=0.05, pk_grid=128),
    # profiling size: particle arrays (16.8M x 26 B) larger than L2, a few GB on the device
    "loop256": dict(layout=dict(ng=256, nnt=2, nns=2, ratio_cs=4, ngb=4, app=0.1), rms=0.5, seed=5200, apm3f=4.0,
                    growth_per_step=0.05, pk_grid=256),
}


def batch_counts(name: str) -> np.ndarray:
    """Lattice side per box of a batch workload: the count N_t = clip(round(median exp(sigma z)))
    of each box (z standard normal, seeded), rounded to the nearest cube m^3."""
    w = WORKLOADS[name]
    nb = w["layout"]["nnt"] ** 3
    rng = np.random.Generator(np.random.PCG64(w["seed"]))
    cnt = np.clip(np.round(w["median"] * np.exp(w["sigma"] * rng.standard_normal(nb))), *w["clip"])
    return np.maximum(np.round(np.cbrt(cnt)).astype(np.int64), 1)


def tile_layout(name: str) -> Layout:
    """One-box layout of a batch workload (the layout each box is cell-sorted with)."""
    w = WORKLOADS[name]
    lw = dict(w["layout"])
    return Layout(ng=w["box"], nnt=1, nns=lw["nns"], ratio_cs=lw["ratio_cs"], ngb=lw["ngb"], app=lw["app"])


def cache_dir() -> str:
    d = os.environ.get("CUBE_WORKLOAD_CACHE", "/tmp/cube2_b200_workloads")
    os.makedirs(d, exist_ok=True)
    return d


def make(name: str, use_cache: bool = True) -> Image:
    """Build (or load from the /tmp cache) the named workload as an Image."""
    w = WORKLOADS[name]
    L = Layout(**w["layout"])
    path = os.path.join(cache_dir(), f"{name}.npz")
    if use_cache and os.path.exists(path):
        z = np.load(path)
        return Image(L, z["xp"], z["vp"], z["rhoc"], z["idx_b_r"], z["pid"], z["active"], int(z["n_particles"]))
    if w["kind"] == "batch":
        boxes = [ic.zeldovich_box(int(m), float(w["box"]), 0.5, w["seed"] + t) for t, m in
                 enumerate(batch_counts(name))]
        img = build_tile_batch(boxes, tile_layout(name), L.nnt)
    else:
        if w["kind"] == "zeldovich":
            pos, vel, _ = ic.zeldovich_lattice(w["n"], w["rms"], w["seed"])
        else:
            pos, vel, _ = ic.lognormal_poisson(w["n"], w["sigma"], w["seed"])
        img = build_image(pos, vel, L)
    if use_cache:
        np.savez(path, xp=img.xp, vp=img.vp, rhoc=img.rhoc, idx_b_r=img.idx_b_r, pid=img.pid, active=img.active,
                 n_particles=img.n_particles)
    return img


def tables(name: str):
    """(isort, ires, ixyz3, apm3, ratio_sf) for a uniform level-2 kick of the workload."""
    w = WORKLOADS[name]
    L = Layout(**w["layout"])
    level = int(np.nonzero(RATIO_SF == w["rsf"])[0][0]) + 1
    return (np.arange(1, L.ns3 + 1, dtype=np.int32), np.full(L.ns3, level, np.int32), ixyz3_table(L),
            apm3_table(w["apm3f"]), RATIO_SF.copy())


def physical_positions(img: Image) -> np.ndarray:
    """Fine-cell positions (float64, decoded fixed point) of each physical particle, indexed by pid."""
    L = img.layout
    nt, ncb, nte = L.nt, L.ncb, L.nte
    flat = img.rhoc.reshape(-1).astype(np.int64)
    t = np.arange(L.nnt)
    e = np.arange(nte) - ncb
    tz, ty, tx, k, j, i = np.meshgrid(t, t, t, e, e, e, indexing="ij")
    g = np.stack([(tx * nt + i).reshape(-1), (ty * nt + j).reshape(-1), (tz * nt + k).reshape(-1)], -1)
    act = np.nonzero(img.active)[0]
    cell = np.repeat(np.arange(flat.size), flat)[act]
    u = img.xp[act].view(np.uint16).astype(np.float64)
    pos = (g[cell] + (u + 0.5) / 65536.0) * L.ratio_cs
    out = np.empty((img.n_particles, 3), np.float64)
    out[img.pid[act]] = np.mod(pos, L.ng)
    return out
