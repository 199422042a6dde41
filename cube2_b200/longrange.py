"""PM1 and PM2, the long-range layers of the reference's force split (cube_pm1_force_device,
cube_pm2_force_device), for a host image: its arrays go to the device (torch tensors as device
memory), the layer kicks vp there, and the kicked vp comes back.

With the periodic PM3 geometry (CUBE_PM3_PERIODIC) the fine mesh already carries the whole
periodic force and these layers are not needed; they complete the split of the reference's own
geometry (CUBE_PM3_SUBTILE meshes with range-limited Green tables): PM1 (coarse, periodic) +
PM2 (tile, range apm1) + PM3 (subtile, range apm2f) + PP (range apm3).
"""
from __future__ import annotations

import ctypes

import numpy as np

from .kick import CUBE_PM3_SUBTILE, FineKick, _check, lib
from .layout import Image


def _dp(t):
    return ctypes.c_void_p(t.data_ptr())


def _run(img: Image, layer: int, args, pm3_mode: int):
    import torch
    FineKick(img.layout, pm3_mode=pm3_mode).configure()
    dev = torch.device("cuda", torch.cuda.current_device())

    def up(a):
        return torch.from_numpy(np.ascontiguousarray(a).reshape(-1).copy()).to(dev)
    rho, idx, xp, vp = up(img.rhoc), up(img.idx_b_r), up(img.xp), up(img.vp)
    f2 = ctypes.c_float()
    vmax = (ctypes.c_float * 3)()
    fn = lib().cube_pm1_force_device if layer == 1 else lib().cube_pm2_force_device
    fargs = [ctypes.c_float(a) for a in args]
    _check(fn(_dp(rho), _dp(idx), _dp(xp), ctypes.c_int64(img.n_used), _dp(vp), *fargs, ctypes.byref(f2), vmax, None),
           f"cube_pm{layer}_force_device")
    torch.cuda.synchronize()
    return vp.cpu().numpy().reshape(-1, 3), float(f2.value), np.array(vmax[:], np.float32)


def pm1_force(img: Image, apm1c: float, mass: float, a_mid: float, dt: float, pm3_mode: int = CUBE_PM3_SUBTILE):
    """PM1 kick of a host image: (vp, f2max, vmax)."""
    return _run(img, 1, (mass, a_mid, dt, apm1c), pm3_mode)


def pm2_force(img: Image, apm2: float, apm1: float, mass: float, a_mid: float, dt: float,
              pm3_mode: int = CUBE_PM3_SUBTILE):
    """PM2 kick of a host image: (vp, f2max, vmax)."""
    return _run(img, 2, (mass, a_mid, dt, apm2, apm1), pm3_mode)
