"""Host-side data formats on either side of the fine-scale kick.

CUBE2 stores particles cell-sorted per tile with a periodic buffer of ``ncb``
coarse cells around each tile (``buffer_particle.f90:23-345``):

* ``xp``      int16 [n_used][3]  fixed-point offset inside the coarse cell
  (``variables.f90:24``; decode ``kick.f90:292``: pos = cell-1 + (u+0.5)/2^16,
  u = (uint16)xp, ``parameters.f90:87-88,118``)
* ``vp``      float32 [n_used][3] velocity (``variables.f90:25``)
* ``rhoc``    int32 C view [tz][ty][tx][k][j][i] over the extended tile,
  nte = nt + 2 ncb cells per side (``variables.f90:26``, ``spine_image``)
* ``idx_b_r`` int64 C view [tz][ty][tx][k][j]: running particle count at the
  end of row (j,k) of tile (tx,ty,tz), tiles in z-major order
  (``variables.f90:146-216`` spine_image)

Particles of coarse cell (i,j,k) of a tile start at
``idx_b_r[..][k][j] - sum(rhoc[..][k][j][i:])`` (``pp_force_kernel.c:203-209``).

This module builds that layout from plain positions (the role of ``buffer_x``
plus ``spine_image`` for a single image), restates the subtile
classification of ``kick.f90:107-131`` and the subtile index table of
``initialize.f90:207-224``.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass(frozen=True)
class Layout:
    """Compile-time layout of the reference (parameters.f90:17-24,56)."""

    ng: int              # fine cells per image side
    nnt: int             # tiles per image side
    nns: int             # subtiles per tile side
    ratio_cs: int = 4    # fine cells per coarse cell
    ngb: int = 4         # tile buffer in fine cells (ncb = ngb / ratio_cs)
    app: float = 0.1     # PP softening in fine cells (parameters.f90:42)

    def __post_init__(self):
        if self.ng % self.ratio_cs or (self.ng // self.ratio_cs) % self.nnt:
            raise ValueError("ng must be divisible by ratio_cs * nnt")
        if (self.ng // self.ratio_cs // self.nnt) % self.nns:
            raise ValueError("nt must be divisible by nns")
        if self.ngb % self.ratio_cs or self.ngb < self.ratio_cs:
            raise ValueError("ngb must be a positive multiple of ratio_cs")

    @property
    def nc(self) -> int:
        return self.ng // self.ratio_cs

    @property
    def nt(self) -> int:
        return self.nc // self.nnt

    @property
    def ntt(self) -> int:
        return self.nt // self.nns

    @property
    def ncb(self) -> int:
        return self.ngb // self.ratio_cs

    @property
    def nte(self) -> int:
        return self.nt + 2 * self.ncb

    @property
    def ns3(self) -> int:
        return (self.nnt * self.nns) ** 3

    def as_dict(self) -> dict:
        return dict(ng=self.ng, nnt=self.nnt, nns=self.nns, ratio_cs=self.ratio_cs, ngb=self.ngb,
                    app=self.app)


# parameters.f90:22 and :38-41 at the reference defaults
RATIO_SF = np.array([1, 2, 4, 6, 8, 12, 16], dtype=np.int32)


def apm3_table(apm3f: float) -> np.ndarray:
    """PP range per level, apm3 = apm3f / ratio_sf (parameters.f90:40)."""
    return (np.float32(apm3f) / RATIO_SF.astype(np.float32)).astype(np.float32)


@dataclass
class Image:
    """One image in the reference layout (arrays in C views, see module doc)."""

    layout: Layout
    xp: np.ndarray        # int16 [n_used, 3]
    vp: np.ndarray        # float32 [n_used, 3]
    rhoc: np.ndarray      # int32 [nnt, nnt, nnt, nte, nte, nte]
    idx_b_r: np.ndarray   # int64 [nnt, nnt, nnt, nte, nte]
    pid: np.ndarray       # int64 [n_used]: index of the source particle
    active: np.ndarray    # bool [n_used]: stored copy lies in the tile interior
    n_particles: int      # physical particles in the image
    extras: dict = field(default_factory=dict)

    @property
    def n_used(self) -> int:
        return int(self.xp.shape[0])


def encode_positions(pos: np.ndarray, ratio_cs: int, nc: int):
    """Fine-cell positions in [0, nc*ratio_cs) -> (coarse cell int64[N,3], u uint16[N,3]).

    Inverse of the decode at kick.f90:292 (writer side: utilities/ic.f90:603,
    ``xp = floor(x / x_resolution)``): u = floor(frac * 2^16).
    """
    x = np.asarray(pos, dtype=np.float64) / ratio_cs
    x = np.mod(x, nc)
    cc = np.floor(x).astype(np.int64)
    frac = x - cc
    u = np.floor(frac * 65536.0).astype(np.int64)
    u = np.clip(u, 0, 65535)
    cc = np.clip(cc, 0, nc - 1)
    return cc, u.astype(np.uint16)


def decode_positions(cell_minus_1: np.ndarray, xp: np.ndarray) -> np.ndarray:
    """kick.f90:292 decode, exact in float64: (cell-1) + (u + 0.5) / 65536."""
    u = xp.astype(np.int16).view(np.uint16).astype(np.float64)
    return cell_minus_1.astype(np.float64) + (u + 0.5) / 65536.0


def build_image(pos: np.ndarray, vel: np.ndarray, layout: Layout) -> Image:
    """Cell-sort particles into the reference's per-tile layout with periodic buffers."""
    L = layout
    nc, nt, ncb, nte, nnt = L.nc, L.nt, L.ncb, L.nte, L.nnt
    cc, u = encode_positions(pos, L.ratio_cs, nc)
    gcell = (cc[:, 2] * nc + cc[:, 1]) * nc + cc[:, 0]
    order = np.argsort(gcell, kind="stable")
    counts = np.bincount(gcell, minlength=nc ** 3).astype(np.int64)
    starts = np.cumsum(counts) - counts

    # global coarse cell of every extended cell, storage order [tz][ty][tx][k][j][i]
    t = np.arange(nnt)
    e = np.arange(nte) - ncb
    tz, ty, tx, k, j, i = np.meshgrid(t, t, t, e, e, e, indexing="ij")
    gx = np.mod(tx * nt + i, nc)
    gy = np.mod(ty * nt + j, nc)
    gz = np.mod(tz * nt + k, nc)
    gext = ((gz * nc + gy) * nc + gx).reshape(-1)
    rhoc_flat = counts[gext]
    total = int(rhoc_flat.sum())
    seg_off = np.cumsum(rhoc_flat) - rhoc_flat
    src = np.repeat(starts[gext] - seg_off, rhoc_flat) + np.arange(total, dtype=np.int64)
    pid = order[src]

    interior = ((i >= 0) & (i < nt) & (j >= 0) & (j < nt) & (k >= 0) & (k < nt)).reshape(-1)
    active = np.repeat(interior, rhoc_flat)

    xp = u[pid].view(np.int16).copy()
    vp = np.ascontiguousarray(np.asarray(vel, dtype=np.float32)[pid])
    rhoc = rhoc_flat.astype(np.int32).reshape(nnt, nnt, nnt, nte, nte, nte)
    idx_b_r = np.cumsum(rhoc.sum(axis=-1, dtype=np.int64).reshape(-1)).reshape(nnt, nnt, nnt, nte, nte)
    return Image(L, xp, vp, rhoc, idx_b_r.astype(np.int64), pid.astype(np.int64), active,
                 n_particles=int(np.asarray(pos).shape[0]))


def build_tile_batch(boxes, tile: Layout, nnt: int) -> Image:
    """A batch of nnt^3 independent periodic boxes as one image of nnt^3 parent tiles.

    ``boxes`` is a list of (pos, vel) per box, positions in [0, tile.ng)^3, in tile order
    t = (tz*nnt + ty)*nnt + tx.  Every box is cell-sorted with ``build_image`` on the one-tile
    layout ``tile`` (so its buffer holds its own periodic copies) and the tiles are stored one
    after the other, with the spine ``idx_b_r`` running over the whole batch.  This is the
    input of the per-tile periodic PM3 geometry (CUBE_PM3_TILE_PERIODIC).  ``pid`` numbers the
    particles of box t after those of boxes 0..t-1.
    """
    if tile.nnt != 1:
        raise ValueError("boxes are laid out with a one-tile layout")
    if len(boxes) != nnt ** 3:
        raise ValueError("need nnt^3 boxes")
    L = Layout(ng=tile.ng * nnt, nnt=nnt, nns=tile.nns, ratio_cs=tile.ratio_cs, ngb=tile.ngb, app=tile.app)
    imgs = [build_image(p, v, tile) for p, v in boxes]
    nte = tile.nte
    xp = np.concatenate([im.xp for im in imgs])
    vp = np.concatenate([im.vp for im in imgs])
    rhoc = np.stack([im.rhoc.reshape(nte, nte, nte) for im in imgs]).reshape(nnt, nnt, nnt, nte, nte, nte)
    offs = np.cumsum([0] + [im.n_used for im in imgs])
    idx = np.stack([im.idx_b_r.reshape(nte, nte) + offs[t] for t, im in enumerate(imgs)])
    poffs = np.cumsum([0] + [im.n_particles for im in imgs])
    pid = np.concatenate([im.pid + poffs[t] for t, im in enumerate(imgs)])
    active = np.concatenate([im.active for im in imgs])
    return Image(L, xp, vp, rhoc.astype(np.int32), idx.reshape(nnt, nnt, nnt, nte, nte).astype(np.int64),
                 pid.astype(np.int64), active, n_particles=int(poffs[-1]))


def ixyz3_table(layout: Layout) -> np.ndarray:
    """Subtile index table (initialize.f90:207-224): rows [sx,sy,sz,tx,ty,tz], 1-based."""
    nnt, nns = layout.nnt, layout.nns
    rows = []
    for tz in range(1, nnt + 1):
        for ty in range(1, nnt + 1):
            for tx in range(1, nnt + 1):
                for sz in range(1, nns + 1):
                    for sy in range(1, nns + 1):
                        for sx in range(1, nns + 1):
                            rows.append((sx, sy, sz, tx, ty, tz))
    return np.array(rows, dtype=np.int32)


def indexed_sort(arr: np.ndarray) -> np.ndarray:
    """Heap-sort index (kick.f90:570-614), ascending; returns 1-based indices."""
    a = np.asarray(arr, dtype=np.float32)
    n = a.shape[0]
    indx = list(range(1, n + 1))
    if n < 2:
        return np.array(indx, dtype=np.int32)
    L = n // 2 + 1
    ir = n
    A = lambda idx: a[idx - 1]  # noqa: E731
    while True:
        if L > 1:
            L -= 1
            indxt = indx[L - 1]
            q = A(indxt)
        else:
            indxt = indx[ir - 1]
            q = A(indxt)
            indx[ir - 1] = indx[0]
            ir -= 1
            if ir == 1:
                indx[0] = indxt
                return np.array(indx, dtype=np.int32)
        i = L
        jj = L + L
        while jj <= ir:
            if jj < ir and A(indx[jj - 1]) < A(indx[jj]):
                jj += 1
            if q < A(indx[jj - 1]):
                indx[i - 1] = indx[jj - 1]
                i = jj
                jj = jj + jj
            else:
                jj = ir + 1
        indx[i - 1] = indxt


def classify_subtiles(rhoc: np.ndarray, layout: Layout):
    """PM3 level per subtile and heavy-first order (kick.f90:107-131).

    npc_max = max(rhoc over the subtile's interior cells) / 64; thresholds
    24 / 114 / 320 / 1350 give ires 2..6.  Returns (ires int32[ns3], isort int32[ns3], 1-based).
    """
    L = layout
    ix = ixyz3_table(L)
    ncb, ntt = L.ncb, L.ntt
    npc = np.zeros(L.ns3, dtype=np.float32)
    ires = np.zeros(L.ns3, dtype=np.int32)
    for it, (sx, sy, sz, tx, ty, tz) in enumerate(ix):
        blk = rhoc[tz - 1, ty - 1, tx - 1,
                   ncb + (sz - 1) * ntt: ncb + sz * ntt,
                   ncb + (sy - 1) * ntt: ncb + sy * ntt,
                   ncb + (sx - 1) * ntt: ncb + sx * ntt]
        v = np.float32(blk.max()) / np.float32(64.0)
        npc[it] = v
        if v < 24:
            ires[it] = 2
        elif v < 114:
            ires[it] = 3
        elif v < 320:
            ires[it] = 4
        elif v < 1350:
            ires[it] = 5
        else:
            ires[it] = 6
    isort = indexed_sort(-npc)
    return ires, isort
