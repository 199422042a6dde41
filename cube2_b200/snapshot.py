"""Checkpoint files of one image (cube_snapshot_write / cube_snapshot_read).

The reference writes, per image, ``<opath>image<i>/<z>_<name>_<i>.bin`` for name in info, xp,
vp, np and id (checkpoint.f90:11-38; names from basic_functions.f08:60-86), right after a
drift, when its arrays hold the physical particles only.  ``write`` takes an image with its
buffers and writes its physical particles in that order; ``read`` reads them back and rebuilds
the buffers with a drift of zero length (cube_drift with dt_mid = 0: every particle stays in
its cell, and the buffer copies are made as after any drift).
"""
from __future__ import annotations

import ctypes

import numpy as np

from .drift import drift_host
from .kick import CUBE_PM3_PERIODIC, FineKick, _check, _p, lib
from .layout import Image, Layout

HEADER_INTS = ("nplocal", "npglobal", "izipx", "izipv", "image", "nn", "nnt", "nt", "ncell", "ncb", "timestep",
               "cur_checkpoint", "cur_halofind")
HEADER_REALS = ("a", "t", "tau", "dt_pp", "dt_pm3", "dt_pm2", "dt_pm1", "dt_vmax", "mass_p_cdm", "box", "h0",
                "omega_m", "omega_l", "s8", "vsim2phys", "sigma_vres", "sigma_vi", "z_i", "vz_max")
HEADER_BYTES = 13 * 8 + 19 * 4


class CSimHeader(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in HEADER_INTS] + [(n, ctypes.c_float) for n in HEADER_REALS]


def file_names(opath: str, image: int, z: float) -> tuple[str, str]:
    """(prefix, suffix) of the reference's output names: prefix = opath + 'image<i>/' + z as
    Fortran f7.3 without blanks + '_', suffix = '_<i>.bin' (basic_functions.f08:60-86)."""
    return f"{opath}image{image}/{z:7.3f}".replace(" ", "") + "_", f"_{image}.bin"


def default_header(L: Layout, nn: int = 1, image: int = 1) -> dict:
    h = {n: 0 for n in HEADER_INTS}
    h.update({n: 0.0 for n in HEADER_REALS})
    h.update(izipx=2, izipv=2, image=image, nn=nn, nnt=L.nnt, nt=L.nt, ncell=L.ratio_cs, ncb=L.ncb, a=1.0,
             mass_p_cdm=1.0)
    return h


def _to_c(h: dict) -> CSimHeader:
    c = CSimHeader()
    for n in HEADER_INTS + HEADER_REALS:
        setattr(c, n, h[n])
    return c


def write(img: Image, prefix: str, suffix: str, header: dict | None = None, pm3_mode: int = CUBE_PM3_PERIODIC):
    """cube_snapshot_write of a host image; nplocal and npglobal default to its physical count."""
    L = img.layout
    FineKick(L, pm3_mode=pm3_mode).configure()
    h = dict(default_header(L) if header is None else header)
    if not h.get("npglobal"):
        h["npglobal"] = img.n_particles
    c = _to_c(h)
    _check(lib().cube_snapshot_write(prefix.encode(), suffix.encode(), ctypes.byref(c),
                                     _p(np.ascontiguousarray(img.rhoc, np.int32)),
                                     _p(np.ascontiguousarray(img.idx_b_r, np.int64)),
                                     _p(np.ascontiguousarray(img.xp, np.int16)),
                                     _p(np.ascontiguousarray(img.vp, np.float32)),
                                     _p(np.ascontiguousarray(img.pid, np.int64)) if img.pid is not None else None),
           "cube_snapshot_write")


def read_physical(L: Layout, prefix: str, suffix: str, with_pid: bool = True, pm3_mode: int = CUBE_PM3_PERIODIC):
    """cube_snapshot_read: (header dict, physical counts [nnt^3][nt][nt][nt], xp, vp, pid or None)."""
    FineKick(L, pm3_mode=pm3_mode).configure()
    c = CSimHeader()
    rc = lib().cube_snapshot_read(prefix.encode(), suffix.encode(), ctypes.byref(c), None, None, None, None,
                                  ctypes.c_int64(0))
    if rc not in (0, 5):  # 5: capacity 0 is too small, the header is filled
        _check(rc, "cube_snapshot_read")
    n = int(c.nplocal)
    rhoc = np.zeros((L.nnt ** 3, L.nt, L.nt, L.nt), np.int32)
    xp = np.zeros((n, 3), np.int16)
    vp = np.zeros((n, 3), np.float32)
    pid = np.zeros(n, np.int64) if with_pid else None
    _check(lib().cube_snapshot_read(prefix.encode(), suffix.encode(), ctypes.byref(c), _p(rhoc), _p(xp), _p(vp),
                                    _p(pid) if with_pid else None, ctypes.c_int64(n)), "cube_snapshot_read")
    h = {name: getattr(c, name) for name in HEADER_INTS + HEADER_REALS}
    return h, rhoc, xp, vp, pid


def read(L: Layout, prefix: str, suffix: str, with_pid: bool = True, pm3_mode: int = CUBE_PM3_PERIODIC):
    """(Image with its buffers rebuilt, header dict)."""
    h, phys, xp, vp, pid = read_physical(L, prefix, suffix, with_pid, pm3_mode)
    nnt, nte, nt, ncb = L.nnt, L.nte, L.nt, L.ncb
    rhoc = np.zeros((nnt, nnt, nnt, nte, nte, nte), np.int32)
    rhoc[:, :, :, ncb:ncb + nt, ncb:ncb + nt, ncb:ncb + nt] = phys.reshape(nnt, nnt, nnt, nt, nt, nt)
    idx = np.cumsum(rhoc.sum(axis=-1, dtype=np.int64).reshape(-1)).reshape(nnt, nnt, nnt, nte, nte)
    n = xp.shape[0]
    bare = Image(L, xp, vp, rhoc, idx, pid if pid is not None else np.arange(n, dtype=np.int64),
                 np.ones(n, bool), n_particles=n)
    return drift_host(bare, 0.0, 0.0, pm3_mode=pm3_mode), h
