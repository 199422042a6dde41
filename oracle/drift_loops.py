"""ORACLE -- test infrastructure only.

A line-by-line restatement, with the reference's loops, of one drift of one image and
the rebuild of its buffers, for small images: ``drift.f90:1-161`` (layer loop,
``rhoce`` / ``rholocal`` counters, ``spine_tile`` of ``variables.f90:124-164``, the
physical-row copy), then ``buffer_grid.f90:13-45`` (``buffer_np``),
``buffer_grid.f90:77-155`` (``redistribute_cdm`` with ``spine_image`` of
``variables.f90:166-216``) and ``buffer_particle.f90:23-345`` (``buffer_xvp``), with one
image (``nn = 1``: every co-indexed array is the image's own).  It pins the vectorised
restatement in ``drift_oracle.py``; the reference itself is Fortran and there is no
Fortran compiler here.

Fortran arrays are kept in their C views: ``rhoc[tz][ty][tx][k][j][i]`` with extended
index ``c = i + ncb - 1``, ``idx_b_r[tz][ty][tx][k][j]``; particle indices are 1-based
where the reference's are.
"""
import numpy as np

from .drift_oracle import nint_half_away, nlayer


def _drift_tile(L, rc, ib, xp, vp, pid, dt_mid, nl):
    """drift.f90:31-150 for one tile: (physical rhoce, compacted x, v, pid of the tile)."""
    nt, ncb = L.nt, L.ncb
    lo, hi = 1 - ncb, nt + ncb
    off = 2 * ncb - 1  # rhoce(1-2ncb : nt+2ncb) -> 0-based
    ne = nt + 4 * ncb
    rhoce = np.zeros((ne, ne, ne), np.int64)
    rholocal = np.zeros((ne, ne, ne), np.int64)
    dt32 = np.float32(dt_mid)
    rcs32 = np.float32(L.ratio_cs)

    def visit():
        for ilayer in range(nl):
            for k in range(lo + ilayer, hi + 1, nl):
                for j in range(lo, hi + 1):
                    for i in range(lo, hi + 1):
                        n = int(rc[k + ncb - 1, j + ncb - 1, i + ncb - 1])
                        nzero = int(ib[k + ncb - 1, j + ncb - 1]) - int(rc[k + ncb - 1, j + ncb - 1, i + ncb - 1:].sum())
                        for l in range(1, n + 1):
                            ip = nzero + l
                            u = xp[ip - 1].view(np.uint16).astype(np.float64)
                            xq = np.array([i, j, k], np.float64) - 1.0 + (u + 0.5) * (1.0 / 65536.0)
                            dtv = (dt32 * vp[ip - 1]).astype(np.float32)
                            deltax = (dtv / rcs32).astype(np.float32)
                            ig = np.ceil(xq + deltax.astype(np.float64)).astype(np.int64)
                            yield ip, ig, dtv

    for ip, ig, _ in visit():  # density loop, drift.f90:38-79
        assert np.all(ig + off >= 0) and np.all(ig + off < ne), "displacement beyond the reference's rhoce"
        rhoce[ig[2] + off, ig[1] + off, ig[0] + off] += 1
    # spine_tile, variables.f90:124-164
    idx_ex_r = np.cumsum(rhoce.sum(axis=2).reshape(-1)).reshape(ne, ne)  # [k][j]
    pp_l = np.zeros((nt, nt), np.int64)
    pp_r = np.zeros((nt, nt), np.int64)
    ppe_l = np.zeros((nt, nt), np.int64)
    ppe_r = np.zeros((nt, nt), np.int64)
    nsum = 0
    for igz in range(1, nt + 1):
        for igy in range(1, nt + 1):
            row = rhoce[igz + off, igy + off]
            ppe_r[igz - 1, igy - 1] = idx_ex_r[igz + off, igy + off] - row[nt + 1 + off:].sum()
            pp_l[igz - 1, igy - 1] = nsum + 1
            np_phy = int(row[1 + off:nt + 1 + off].sum())
            nsum += np_phy
            pp_r[igz - 1, igy - 1] = nsum
            ppe_l[igz - 1, igy - 1] = ppe_r[igz - 1, igy - 1] - np_phy + 1
    n_ext = int(idx_ex_r[-1, -1])
    xp_new = np.zeros((n_ext, 3), np.int16)
    vp_new = np.zeros((n_ext, 3), np.float32)
    pid_new = np.zeros(n_ext, np.int64)
    for ip, ig, dtv in visit():  # drift.f90:82-118
        a, b, c = ig[2] + off, ig[1] + off, ig[0] + off
        rholocal[a, b, c] += 1
        idx = int(idx_ex_r[a, b]) - int(rhoce[a, b, c:].sum()) + int(rholocal[a, b, c])
        step = nint_half_away(dtv.astype(np.float64) / (np.float64(2.0 ** -16) * L.ratio_cs))
        xp_new[idx - 1] = ((xp[ip - 1].astype(np.int64) + step) & 0xFFFF).astype(np.uint16).view(np.int16)
        vp_new[idx - 1] = vp[ip - 1]
        if pid is not None:
            pid_new[idx - 1] = pid[ip - 1]
    # delete particles, drift.f90:121-133
    n_phys = int(pp_r[nt - 1, nt - 1])
    x = np.zeros((n_phys, 3), np.int16)
    v = np.zeros((n_phys, 3), np.float32)
    p = np.zeros(n_phys, np.int64)
    for k in range(nt):
        for j in range(nt):
            d0, d1, s0 = pp_l[k, j] - 1, pp_r[k, j], ppe_l[k, j] - 1
            x[d0:d1] = xp_new[s0:s0 + d1 - d0]
            v[d0:d1] = vp_new[s0:s0 + d1 - d0]
            p[d0:d1] = pid_new[s0:s0 + d1 - d0]
    phys = rhoce[1 + off:nt + 1 + off, 1 + off:nt + 1 + off, 1 + off:nt + 1 + off]
    return phys, x, v, p


def _spine_image(L, rhoc):
    """variables.f90:166-216 on the C view of rhoc; returns dict of [tz][ty][tx][k][j] arrays
    (idx_b_l, idx_b_r) and [tz][ty][tx][igz-1][igy-1] arrays (ppl0, pplr, pprl, ppr0, ppl, ppr)."""
    nt, ncb, nnt = L.nt, L.ncb, L.nnt
    c0 = ncb - 1  # extended index of Fortran 0
    rows = rhoc.sum(axis=-1, dtype=np.int64)  # [t..][k][j]
    tile_tot = rhoc.sum(axis=(3, 4, 5), dtype=np.int64)
    tile_phys = rhoc[:, :, :, ncb:ncb + nt, ncb:ncb + nt, ncb:ncb + nt].sum(axis=(3, 4, 5), dtype=np.int64)
    flat_tot = tile_tot.reshape(-1)
    flat_phys = tile_phys.reshape(-1)
    ctile = (np.cumsum(flat_tot) - flat_tot).reshape(nnt, nnt, nnt)
    ctile_p = (np.cumsum(flat_phys) - flat_phys).reshape(nnt, nnt, nnt)
    incl = np.cumsum(rows.reshape(nnt, nnt, nnt, -1), axis=-1).reshape(rows.shape)
    idx_b_r = incl + ctile[..., None, None]
    idx_b_l = idx_b_r - rows
    s = {}
    phys_rows = rhoc[:, :, :, ncb:ncb + nt, ncb:ncb + nt, ncb:ncb + nt].sum(axis=-1, dtype=np.int64)
    pincl = np.cumsum(phys_rows.reshape(nnt, nnt, nnt, -1), axis=-1).reshape(phys_rows.shape)
    s["ppr"] = pincl + ctile_p[..., None, None]
    s["ppl"] = s["ppr"] - phys_rows
    br = idx_b_r[:, :, :, ncb:ncb + nt, ncb:ncb + nt]
    bl = idx_b_l[:, :, :, ncb:ncb + nt, ncb:ncb + nt]
    rr = rhoc[:, :, :, ncb:ncb + nt, ncb:ncb + nt, :]
    s["ppr0"] = br - rr[..., nt + 1 + c0:].sum(axis=-1)
    s["pprl"] = s["ppr0"] - rr[..., nt - ncb + 1 + c0:nt + 1 + c0].sum(axis=-1)
    s["ppl0"] = bl + rr[..., :1 + c0].sum(axis=-1)
    s["pplr"] = s["ppl0"] + rr[..., 1 + c0:ncb + 1 + c0].sum(axis=-1)
    s["idx_b_l"], s["idx_b_r"] = idx_b_l, idx_b_r
    return s


def _buffer_np(L, rhoc):
    """buffer_grid.f90:13-45 with one image: periodic copies in x, then y, then z."""
    nt, ncb = L.nt, L.ncb
    r = rhoc.copy()
    lo_h, hi_h = slice(0, ncb), slice(ncb + nt, nt + 2 * ncb)
    src_lo, src_hi = slice(nt, nt + ncb), slice(ncb, 2 * ncb)  # (nt-ncb+1:nt) and (1:ncb)
    # x (axis 5; tiles on axis 2)
    r[:, :, :, :, :, lo_h] = np.roll(r[:, :, :, :, :, src_lo], 1, axis=2)
    r[:, :, :, :, :, hi_h] = np.roll(r[:, :, :, :, :, src_hi], -1, axis=2)
    # y (axis 4; tiles on axis 1)
    r[:, :, :, :, lo_h, :] = np.roll(r[:, :, :, :, src_lo, :], 1, axis=1)
    r[:, :, :, :, hi_h, :] = np.roll(r[:, :, :, :, src_hi, :], -1, axis=1)
    # z (axis 3; tiles on axis 0)
    r[:, :, :, lo_h, :, :] = np.roll(r[:, :, :, src_lo, :, :], 1, axis=0)
    r[:, :, :, hi_h, :, :] = np.roll(r[:, :, :, src_hi, :, :], -1, axis=0)
    return r


def _buffer_xvp(L, s, arr):
    """buffer_particle.f90:23-345 (x, then y, then z copies) on one array, in place."""
    nt, ncb, nnt = L.nt, L.ncb, L.nnt
    bl, br = s["idx_b_l"], s["idx_b_r"]
    e = lambda f: f + ncb - 1  # noqa: E731  Fortran index -> extended index
    for tz in range(nnt):
        for ty in range(nnt):
            for tx in range(nnt):
                sx = (tx - 1) % nnt
                for iz in range(nt):
                    for iy in range(nt):
                        d0, d1 = bl[tz, ty, tx, e(iz + 1), e(iy + 1)], s["ppl0"][tz, ty, tx, iz, iy]
                        s0, s1 = s["pprl"][tz, ty, sx, iz, iy], s["ppr0"][tz, ty, sx, iz, iy]
                        arr[d0:d1] = arr[s0:s1]
    for tz in range(nnt):
        for ty in range(nnt):
            for tx in range(nnt):
                sx = (tx + 1) % nnt
                for iz in range(nt):
                    for iy in range(nt):
                        d0, d1 = s["ppr0"][tz, ty, tx, iz, iy], br[tz, ty, tx, e(iz + 1), e(iy + 1)]
                        s0, s1 = s["ppl0"][tz, ty, sx, iz, iy], s["pplr"][tz, ty, sx, iz, iy]
                        arr[d0:d1] = arr[s0:s1]
    for tz in range(nnt):
        for ty in range(nnt):
            for tx in range(nnt):
                sy = (ty - 1) % nnt
                for iz in range(1, nt + 1):
                    d0, d1 = bl[tz, ty, tx, e(iz), e(1 - ncb)], br[tz, ty, tx, e(iz), e(0)]
                    s0, s1 = bl[tz, sy, tx, e(iz), e(nt - ncb + 1)], br[tz, sy, tx, e(iz), e(nt)]
                    arr[d0:d1] = arr[s0:s1]
    for tz in range(nnt):
        for ty in range(nnt):
            for tx in range(nnt):
                sy = (ty + 1) % nnt
                for iz in range(1, nt + 1):
                    d0, d1 = bl[tz, ty, tx, e(iz), e(nt + 1)], br[tz, ty, tx, e(iz), e(nt + ncb)]
                    s0, s1 = bl[tz, sy, tx, e(iz), e(1)], br[tz, sy, tx, e(iz), e(ncb)]
                    arr[d0:d1] = arr[s0:s1]
    for tz in range(nnt):
        for ty in range(nnt):
            for tx in range(nnt):
                sz = (tz - 1) % nnt
                d0, d1 = bl[tz, ty, tx, e(1 - ncb), e(1 - ncb)], br[tz, ty, tx, e(0), e(nt + ncb)]
                s0, s1 = bl[sz, ty, tx, e(nt - ncb + 1), e(1 - ncb)], br[sz, ty, tx, e(nt), e(nt + ncb)]
                arr[d0:d1] = arr[s0:s1]
    for tz in range(nnt):
        for ty in range(nnt):
            for tx in range(nnt):
                sz = (tz + 1) % nnt
                d0, d1 = bl[tz, ty, tx, e(nt + 1), e(1 - ncb)], br[tz, ty, tx, e(nt + ncb), e(nt + ncb)]
                s0, s1 = bl[sz, ty, tx, e(1), e(1 - ncb)], br[sz, ty, tx, e(ncb), e(nt + ncb)]
                arr[d0:d1] = arr[s0:s1]


def drift_image_loops(L, rhoc, idx_b_r, xp, vp, pid, dt_mid: float, vz_max: float):
    """drift, buffer_grid, buffer_x and buffer_v as the reference sequences them (main.f90:26-31):
    (rhoc, idx_b_r, xp, vp, pid, n_physical)."""
    nt, ncb, nnt = L.nt, L.ncb, L.nnt
    nl = nlayer(dt_mid, vz_max, L.ratio_cs)
    rhoc_new = np.zeros_like(rhoc)
    xs, vs, ps = [], [], []
    for tz in range(nnt):
        for ty in range(nnt):
            for tx in range(nnt):
                phys, x, v, p = _drift_tile(L, rhoc[tz, ty, tx], idx_b_r[tz, ty, tx], xp, vp, pid, dt_mid, nl)
                rhoc_new[tz, ty, tx, ncb:ncb + nt, ncb:ncb + nt, ncb:ncb + nt] = phys
                xs.append(x)
                vs.append(v)
                ps.append(p)
    xphys, vphys, pphys = np.concatenate(xs), np.concatenate(vs), np.concatenate(ps)
    rhoc_new = _buffer_np(L, rhoc_new)
    s = _spine_image(L, rhoc_new)
    n_ext = int(s["idx_b_r"][-1, -1, -1, -1, -1])
    out_x = np.zeros((n_ext, 3), np.int16)
    out_v = np.zeros((n_ext, 3), np.float32)
    out_p = np.zeros(n_ext, np.int64)
    for tz in range(nnt):  # redistribute_cdm, buffer_grid.f90:131-146
        for ty in range(nnt):
            for tx in range(nnt):
                for iz in range(nt):
                    for iy in range(nt):
                        d0, d1 = s["ppl0"][tz, ty, tx, iz, iy], s["ppr0"][tz, ty, tx, iz, iy]
                        s0 = s["ppl"][tz, ty, tx, iz, iy]
                        out_x[d0:d1] = xphys[s0:s0 + d1 - d0]
                        out_v[d0:d1] = vphys[s0:s0 + d1 - d0]
                        out_p[d0:d1] = pphys[s0:s0 + d1 - d0]
    for a in (out_x, out_v, out_p):
        _buffer_xvp(L, s, a)
    return rhoc_new, s["idx_b_r"], out_x, out_v, (out_p if pid is not None else None), int(xphys.shape[0])
