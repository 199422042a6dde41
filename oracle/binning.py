"""ORACLE -- test infrastructure only.  numpy restatement of the reference PP binning.

Restates pp_force_kernel.c:196-274 for one parent tile:
  keys (pp_force_kernel.c:213-236): xvec = (float)((i-ncb) + (u+0.5)/2^16),
      idx = floor((float)rcp * xvec) + rcp, key = (idx2*S + idx1)*S + idx0;
  radix_sort_u32_pair (:76-132): stable sort of (key, slot);
  cell_start (:258-274): first slot of each key, empty cells take the next start.
Checked against the reference's own arrays (golden fixtures) by the tests.
"""
from __future__ import annotations

import numpy as np


def bin_tile(img, tile_xyz, rcp: int):
    """Return dict(keys, values, cell_start, xf_sorted [3][N], ip_local) like the reference."""
    L = img.layout
    nt, ncb = L.nt, L.ncb
    tx, ty, tz = tile_xyz
    rhoc = img.rhoc[tz, ty, tx].astype(np.int64)
    row_end = img.idx_b_r[tz, ty, tx]
    suffix = np.flip(np.cumsum(np.flip(rhoc, -1), -1), -1)  # sum(rhoc[k][j][i:])
    npgrid = nt * rcp
    S = npgrid + 2 * rcp
    lo, hi = ncb - 1, ncb + nt  # region cells (pp_force_kernel.c:199-201)
    reg = rhoc[lo:hi + 1, lo:hi + 1, lo:hi + 1]
    kk, jj, ii = np.nonzero(reg)  # C order = the reference's (k, j, i) loop order
    kk, jj, ii = kk + lo, jj + lo, ii + lo
    cnt = rhoc[kk, jj, ii]
    nzero = row_end[kk, jj] - suffix[kk, jj, ii]
    N = int(cnt.sum())
    seg = np.cumsum(cnt) - cnt
    ip_local = np.repeat(nzero - seg, cnt) + np.arange(N, dtype=np.int64)
    c = np.stack([ii - ncb, jj - ncb, kk - ncb], -1).astype(np.float64)
    c = np.repeat(c, cnt, axis=0)
    u = img.xp[ip_local].view(np.uint16).astype(np.float64)
    x = (c + (u + 0.5) * (1.0 / 65536.0)).astype(np.float32)
    idx = np.floor(np.float32(rcp) * x).astype(np.int64) + rcp
    keys = ((idx[:, 2] * S + idx[:, 1]) * S + idx[:, 0]).astype(np.uint32)
    order = np.argsort(keys, kind="stable")
    skeys = keys[order]
    grid = S ** 3
    big = np.iinfo(np.int64).max
    cs = np.full(grid + 1, big, np.int64)
    first = np.ones(skeys.shape[0], bool)
    first[1:] = skeys[1:] != skeys[:-1]
    cs[skeys[first].astype(np.int64)] = np.nonzero(first)[0]
    cs[grid] = N
    cs = np.minimum.accumulate(cs[::-1])[::-1]
    xf = (np.float32(L.ratio_cs) * x).astype(np.float32)
    return dict(keys=skeys, values=order.astype(np.uint32), cell_start=cs.astype(np.int32),
                xf_sorted=np.ascontiguousarray(xf[order].T), ip_local=ip_local)
