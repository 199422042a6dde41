"""Generate the golden fixtures of tests/golden/ (run on a machine with the reference tree).

The reference ships no tests or golden vectors, so the fixtures are produced
by the reference's own CPU PP kernel (pp_force_kernel.c, compiled from its
source by oracle/build_ref.py) on small seeded inputs:

* ``pp_<case>.npz``: the inputs in the reference layout (xp, vp, rhoc,
  idx_b_r), the reference's kick (vp after c_pp_force_kernel with
  a_mid*dt = 6*pi so that dv equals the force, f2max, vmax, ptotal) and the
  internal arrays of c_pp_force_kernel_tile for every parent tile (sorted
  keys, values, cell_start, sorted positions, ip_local, forces).
* ``green_<n>.npz``: Green_3D tables from the FP64 restatement
  (oracle/pm3_oracle.c) for small meshes, pinned here so later edits of the
  restatement are caught.
* ``fra.npz``: the reference F_ra (pp_force_kernel.c:45-74) on a grid of r.

Usage: python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

from cube2_b200 import ic  # noqa: E402
from cube2_b200.layout import RATIO_SF, Layout, apm3_table, build_image  # noqa: E402
from oracle import oracle as O  # noqa: E402
from oracle.layouts import LAYOUTS  # noqa: E402

SIXPI = np.float32(6 * np.pi)


def _edge_positions(L: Layout, seed: int) -> np.ndarray:
    """Uniform particles plus edge cases: a crowded coarse cell, fixed-point extremes
    u = 0 and u = 65535 next to tile faces, coincident pairs, an empty region."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = L.ng
    pos = [rng.random((n ** 3 // 8, 3)) * n]
    # crowded coarse cell (occupancy far above the mean)
    pos.append(rng.random((300, 3)) * L.ratio_cs + np.array([L.ratio_cs] * 3))
    # fixed-point extremes on every coarse-cell face of one row
    lo = np.array([[c * L.ratio_cs + 0.0, 1.0, 2.0] for c in range(L.nc)])
    hi = np.array([[(c + 1) * L.ratio_cs - L.ratio_cs / 65536.0 * 0.5, 1.0, 2.0] for c in range(L.nc)])
    pos += [lo, hi]
    # coincident pairs (r = 0 is excluded by the reference)
    d = rng.random((20, 3)) * n
    pos += [d, d.copy()]
    pos = np.concatenate(pos)
    # empty slab: drop everything with z in [n/2, n/2 + ratio_cs)
    keep = ~((pos[:, 2] >= n / 2) & (pos[:, 2] < n / 2 + L.ratio_cs))
    return np.mod(pos[keep], n)


def make_pp(case: str, layout_name: str, seed: int, edge: bool):
    L = Layout(**LAYOUTS[layout_name])
    if edge:
        pos = _edge_positions(L, seed)
        rng = np.random.Generator(np.random.PCG64(seed + 1))
        vel = (0.05 * rng.standard_normal(pos.shape)).astype(np.float32)
    else:
        pos, vel = ic.uniform_random(L.ng ** 3 // 8, float(L.ng), seed)
    img = build_image(pos, vel, L)
    apm3 = apm3_table(4.0)
    ref = O.RefPP(L)
    vp, f2, vmax, pt = ref.kick(img, [2] * L.nnt ** 3, apm3, RATIO_SF, 1.0, SIXPI, 1.0)
    tiles = {}
    for tz in range(L.nnt):
        for ty in range(L.nnt):
            for tx in range(L.nnt):
                t = (tz * L.nnt + ty) * L.nnt + tx
                cap = ref.tile(img, (tx, ty, tz), 2, apm3, RATIO_SF, 1.0, SIXPI, 1.0, capture=True)
                for k in ("keys", "values", "cell_start", "xf_sorted", "ip_local", "af"):
                    tiles[f"t{t}_{k}"] = cap[k]
    np.savez_compressed(os.path.join(HERE, f"pp_{case}.npz"), layout=np.array(layout_name), xp=img.xp, vp=img.vp,
                        rhoc=img.rhoc, idx_b_r=img.idx_b_r, active=img.active, vp_ref=vp, f2max_ref=f2,
                        vmax_ref=vmax, ptotal_ref=pt, **tiles)
    print(case, "n_used", img.n_used, "f2max", f2)


def make_green():
    for n, soft, rng_, gs in ((16, 4.0, 0.0, 0.5), (24, 4.0, 7.0, 0.5), (20, 3.5, 7.0, 0.25)):
        G = O.green(n, soft, rng_, gs)
        np.savez_compressed(os.path.join(HERE, f"green_{n}.npz"), G=G, n=n, apm_soft=soft, apm_range=rng_,
                            gridsize=gs)
        print("green", n)


def make_fra():
    ref = O.RefPP(Layout(**LAYOUTS["t32"]))
    r = np.linspace(0.0, 3.0, 601, dtype=np.float32)[1:]
    apm = np.array([0.0, 0.06, 0.1, 1.0, 1.75, 2.0], np.float32)
    F = np.array([[ref.F_ra(float(x), float(a)) for x in r] for a in apm], np.float32)
    np.savez_compressed(os.path.join(HERE, "fra.npz"), r=r, apm=apm, F=F)
    print("fra")


if __name__ == "__main__":
    make_pp("t32", "t32", 11, edge=False)
    make_pp("t32_edge", "t32", 12, edge=True)
    make_pp("t32b_edge", "t32b", 13, edge=True)
    make_green()
    make_fra()
