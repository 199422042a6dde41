"""ORACLE -- test infrastructure only.  Direct restatement of the PP pair force with
per-particle ranges (pp_force_kernel.cu:192-250 semantics: the i-particle's own
range apm3(ires of its subtile)), in float64, with a cKDTree neighbour search.

a_i = sum_{j: 0 < r_ij < rc_i} (x_j - x_i)/r_ij * (F_ra(r_ij, app) - F_ra(r_ij, rc_i))
in fine-cell units over a periodic box (minimum image); used for layouts the
reference CPU kernel cannot express (mixed levels inside one parent tile).
"""
from __future__ import annotations

import numpy as np


def F_ra(r, a):
    """basic_functions.f08:95-109, vectorised in float64."""
    r = np.asarray(r, np.float64)
    a = np.broadcast_to(np.asarray(a, np.float64), r.shape)
    out = np.zeros_like(r)
    with np.errstate(divide="ignore", invalid="ignore"):
        ep = np.where(a > 0, 2 * r / np.where(a > 0, a, 1), np.inf)
        far = (a == 0) | (ep > 2)
        out = np.where(far, 1.0 / (r * r), out)
        o = (~far) & (ep > 1)
        po = (1 / 35 / a ** 2) * (12 / ep ** 2 - 224 + 896 * ep - 840 * ep ** 2 + 224 * ep ** 3 + 70 * ep ** 4
                                  - 48 * ep ** 5 + 7 * ep ** 6)
        out = np.where(o, po, out)
        i = (~far) & (~o) & (ep > 0)
        pi = (1 / 35 / a ** 2) * (224 * ep - 224 * ep ** 3 + 70 * ep ** 4 + 48 * ep ** 5 - 21 * ep ** 6)
        out = np.where(i, pi, out)
    return out


def pp_forces(pos: np.ndarray, box: float, app: float, ranges: np.ndarray) -> np.ndarray:
    """PP accelerations of every particle (float64 [N,3]); ranges[i] = rc of particle i."""
    from scipy.spatial import cKDTree
    pos = np.mod(np.asarray(pos, np.float64), box)
    tree = cKDTree(pos, boxsize=box)
    F = np.zeros_like(pos)
    rmax = float(np.max(ranges))
    pairs = tree.query_pairs(rmax, output_type="ndarray")
    if pairs.size == 0:
        return F
    i = np.concatenate([pairs[:, 0], pairs[:, 1]])
    j = np.concatenate([pairs[:, 1], pairs[:, 0]])
    d = pos[j] - pos[i]
    d -= box * np.round(d / box)
    r = np.sqrt(np.sum(d * d, axis=1))
    rc = ranges[i]
    keep = (r > 0) & (r < rc)
    i, d, r, rc = i[keep], d[keep], r[keep], rc[keep]
    s = (F_ra(r, app) - F_ra(r, rc)) / r
    np.add.at(F, i, d * s[:, None])
    return F
