"""ORACLE -- test infrastructure only.

CPU restatement of one drift of one periodic image followed by the rebuild of its
buffers: ``drift.f90:1-161`` (fixed-point drift, re-binning by coarse cell, compaction
of each tile's physical particles) and then ``buffer_grid.f90:13-45`` (periodic copy of
the cell counts), ``buffer_grid.f90:77-155`` (``redistribute_cdm``: particles moved to
the extended spine) and ``buffer_particle.f90:23-345`` (``buffer_x`` / ``buffer_v``:
every buffer cell receives a copy of the particles of the physical cell it mirrors), for
one image (``nn = 1``: every co-indexed reference is the image itself).

Arithmetic follows the reference's kinds:
- the position of a stored copy is ``xq = (i-1) + (u + 0.5) * 2^-16`` in real(8)
  (``drift.f90:57``), exact;
- ``deltax = (dt_mid * vp) / ratio_cs`` in real(4) (``drift.f90:63``);
- the new coarse cell is ``ceiling(xq + deltax)`` in real(8) (``drift.f90:66``);
- the new offset is ``xp + nint(dt_mid * vp / (x_resolution * ratio_cs))``
  (``drift.f90:111``): a real(4) product divided in real(8), rounded half away from zero,
  added in integer(4) and stored in integer(2) (wrapping modulo 2^16);
- ``nlayer = 2 * ceiling(dt_mid * vz_max / ratio_cs) + 2`` (``drift.f90:26``) in real(4).

Order.  The reference visits a tile's source cells layer by layer (``ilayer`` = the
source row k shifted by ``ncb``, modulo ``nlayer``), then in storage order (k, j, i,
particle), and appends each kept particle to its destination cell
(``drift.f90:94-118``).  Source rows of one layer are at least ``nlayer`` apart, so two
of them never feed the same destination while the z displacement stays below
``nlayer / 2``; the order inside a destination cell is therefore by (ilayer, storage
index).  The restatement sorts by (destination cell, ilayer, storage index), which is
that order, without the loops.  The buffers copy whole cells in order
(``buffer_particle.f90:44-345``), so a buffer cell holds its mirrored cell's particles in
the same order.
"""
import numpy as np


def nlayer(dt_mid: float, vz_max: float, ratio_cs: int) -> int:
    """drift.f90:26 in real(4)."""
    q = np.float32(np.float32(dt_mid) * np.float32(vz_max)) / np.float32(ratio_cs)
    return 2 * int(np.ceil(np.float32(q))) + 2


def nint_half_away(x: np.ndarray) -> np.ndarray:
    """Fortran NINT: nearest integer, halves away from zero (exact in float64 here)."""
    return (np.sign(x) * np.floor(np.abs(x) + 0.5)).astype(np.int64)


def _source_cells(layout, rhoc):
    """Tile and extended cell (cx, cy, cz) of every stored copy, in storage order."""
    nte = layout.nte
    counts = rhoc.reshape(-1).astype(np.int64)
    cell = np.repeat(np.arange(counts.size, dtype=np.int64), counts)
    t, rem = np.divmod(cell, nte ** 3)
    cz, rem = np.divmod(rem, nte * nte)
    cy, cx = np.divmod(rem, nte)
    return t, cx, cy, cz


def drift_physical(layout, rhoc, xp, vp, pid, dt_mid: float, vz_max: float):
    """drift.f90:46-161: the particles each tile keeps, by global destination cell.

    Returns (counts [nc^3] per global coarse cell (z, y, x), xp, vp, pid of the kept
    particles sorted by (cell, ilayer, storage index))."""
    L = layout
    nt, ncb, nnt, nc = L.nt, L.ncb, L.nnt, L.nc
    t, cx, cy, cz = _source_cells(L, rhoc)
    tz, rem = np.divmod(t, nnt * nnt)
    ty, tx = np.divmod(rem, nnt)
    u = np.asarray(xp, np.int16).view(np.uint16).astype(np.float64)
    c = np.stack([cx, cy, cz], axis=1)
    xq = (c - ncb).astype(np.float64) + (u + 0.5) * (1.0 / 65536.0)
    dtv = (np.float32(dt_mid) * np.asarray(vp, np.float32)).astype(np.float32)
    delta = (dtv / np.float32(L.ratio_cs)).astype(np.float32)
    with np.errstate(invalid="ignore"):
        ig = np.ceil(xq + delta.astype(np.float64))
    keep = np.all((ig >= 1) & (ig <= nt), axis=1)
    ig = np.where(keep[:, None], ig, 1).astype(np.int64)
    g = np.stack([tx, ty, tz], axis=1) * nt + ig - 1
    gcell = (g[:, 2] * nc + g[:, 1]) * nc + g[:, 0]
    layer = cz % nlayer(dt_mid, vz_max, L.ratio_cs)
    ip = np.arange(xp.shape[0], dtype=np.int64)
    sel = np.nonzero(keep)[0]
    order = sel[np.lexsort((ip[sel], layer[sel], gcell[sel]))]
    step = nint_half_away(dtv.astype(np.float64) / (np.float64(2.0 ** -16) * L.ratio_cs))
    xp_new = ((np.asarray(xp, np.int16).astype(np.int64) + step) & 0xFFFF).astype(np.uint16).view(np.int16)
    counts = np.bincount(gcell[order], minlength=nc ** 3).astype(np.int64)
    out_pid = None if pid is None else np.asarray(pid)[order]
    return counts, xp_new[order], np.asarray(vp, np.float32)[order], out_pid


def mirrored_cells(layout, tile_periodic: bool = False):
    """Physical cell (z, y, x) of the image mirrored by every extended cell, in storage order
    (buffer_grid.f90:22-40); with tile_periodic every tile is its own periodic box."""
    L = layout
    nc, nt, ncb, nte, nnt = L.nc, L.nt, L.ncb, L.nte, L.nnt
    t = np.arange(nnt)
    e = np.arange(nte) - ncb
    tz, ty, tx, k, j, i = np.meshgrid(t, t, t, e, e, e, indexing="ij")
    if tile_periodic:
        gz, gy, gx = tz * nt + np.mod(k, nt), ty * nt + np.mod(j, nt), tx * nt + np.mod(i, nt)
    else:
        gz, gy, gx = np.mod(tz * nt + k, nc), np.mod(ty * nt + j, nc), np.mod(tx * nt + i, nc)
    phys = ((i >= 0) & (i < nt) & (j >= 0) & (j < nt) & (k >= 0) & (k < nt)).reshape(-1)
    return ((gz * nc + gy) * nc + gx).reshape(-1), phys


def assemble(layout, counts, xp, vp, pid, tile_periodic: bool = False):
    """buffer_grid.f90 + buffer_particle.f90 on one image: the extended layout of
    physical cells `counts` whose particles are (xp, vp, pid) in cell order.
    Returns (rhoc, idx_b_r, xp, vp, pid) of the image with its buffers."""
    L = layout
    nte, nnt = L.nte, L.nnt
    starts = np.cumsum(counts) - counts
    gext, _ = mirrored_cells(L, tile_periodic)
    rhoc_flat = counts[gext]
    seg = np.cumsum(rhoc_flat) - rhoc_flat
    total = int(rhoc_flat.sum())
    src = np.repeat(starts[gext] - seg, rhoc_flat) + np.arange(total, dtype=np.int64)
    rhoc = rhoc_flat.astype(np.int32).reshape(nnt, nnt, nnt, nte, nte, nte)
    idx_b_r = np.cumsum(rhoc.sum(axis=-1, dtype=np.int64).reshape(-1)).reshape(nnt, nnt, nnt, nte, nte)
    return (rhoc, idx_b_r.astype(np.int64), np.ascontiguousarray(xp[src]), np.ascontiguousarray(vp[src]),
            None if pid is None else np.ascontiguousarray(pid[src]))


def drift_image(layout, rhoc, xp, vp, pid, dt_mid: float, vz_max: float, tile_periodic: bool = False):
    """One drift and buffer rebuild: (rhoc, idx_b_r, xp, vp, pid, n_physical)."""
    counts, x, v, p = drift_physical(layout, rhoc, xp, vp, pid, dt_mid, vz_max)
    return (*assemble(layout, counts, x, v, p, tile_periodic), int(counts.sum()))


def buffer_v(layout, rhoc, vp, tile_periodic: bool = False):
    """buffer_particle.f90 buffer_v: every buffer copy takes the velocity of the physical
    particle it mirrors (the kick only updates physical particles)."""
    L = layout
    nc = L.nc
    gext, phys = mirrored_cells(L, tile_periodic)
    counts_ext = rhoc.reshape(-1).astype(np.int64)
    start_ext = np.cumsum(counts_ext) - counts_ext
    owner_start = np.zeros(nc ** 3, np.int64)
    owner_start[gext[phys]] = start_ext[phys]
    total = int(counts_ext.sum())
    within = np.arange(total, dtype=np.int64) - np.repeat(start_ext, counts_ext)
    src = np.repeat(owner_start[gext], counts_ext) + within
    return np.ascontiguousarray(np.asarray(vp, np.float32)[src])
