"""Drift and buffer rebuild on the device (cube_drift_device, cube_drift, cube_buffer_v_device).

One step of the reference's main loop (main.f90:26-31) is drift, buffer_grid, buffer_x,
kick, buffer_v.  ``DeviceImage.drift`` does the first three in one library call and
``DeviceImage.buffer_v`` the last; the kick in between is ``FineKick.kick_fine_device`` on
the same arrays.  The image lives in torch tensors used as device memory only, double
buffered: the drift writes the other buffer and the two swap.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .kick import CUBE_PM3_PERIODIC, CubeError, FineKick, _check, _p, lib
from .layout import Image, Layout

CUBE_ERR_CAPACITY = 5


def _dp(x):
    return ctypes.c_void_p(x if isinstance(x, int) else x.data_ptr())


def _sp(stream):
    return None if stream is None else ctypes.c_void_p(stream if isinstance(stream, int) else stream.cuda_stream)


def drift_host(img: Image, dt_mid: float, vz_max: float, pm3_mode: int = CUBE_PM3_PERIODIC,
               capacity: int | None = None) -> Image:
    """cube_drift on host copies of the image's arrays; returns the drifted image (pid carried,
    `active` recomputed from the new layout)."""
    L = img.layout
    FineKick(L, pm3_mode=pm3_mode).configure()
    cap = int(capacity if capacity is not None else max(2 * img.n_used, 1024))
    n_new, n_phys = ctypes.c_int64(), ctypes.c_int64()
    for attempt in range(2):  # on a capacity error the call reports the size it needs
        rhoc = np.ascontiguousarray(img.rhoc, np.int32).copy()
        idx = np.ascontiguousarray(img.idx_b_r, np.int64).copy()
        xp = np.zeros((cap, 3), np.int16)
        vp = np.zeros((cap, 3), np.float32)
        pid = np.zeros(cap, np.int64)
        xp[:img.n_used] = img.xp
        vp[:img.n_used] = img.vp
        pid[:img.n_used] = img.pid
        st = lib().cube_drift(_p(rhoc), _p(idx), _p(xp), _p(vp), _p(pid), ctypes.c_int64(img.n_used),
                              ctypes.c_int64(cap), ctypes.c_float(dt_mid), ctypes.c_float(vz_max),
                              ctypes.byref(n_new), ctypes.byref(n_phys))
        if st == CUBE_ERR_CAPACITY and attempt == 0 and capacity is None and n_new.value > cap:
            cap = int(n_new.value)
            continue
        _check(st, "cube_drift")
        break
    n = n_new.value
    return Image(L, xp[:n].copy(), vp[:n].copy(), rhoc, idx, pid[:n].copy(), interior_mask(L, rhoc),
                 n_particles=int(n_phys.value))


def interior_mask(L: Layout, rhoc: np.ndarray) -> np.ndarray:
    """Per stored copy: does it lie in its tile's physical region?"""
    nt, ncb, nte = L.nt, L.ncb, L.nte
    e = np.arange(nte) - ncb
    k, j, i = np.meshgrid(e, e, e, indexing="ij")
    inner = ((i >= 0) & (i < nt) & (j >= 0) & (j < nt) & (k >= 0) & (k < nt)).reshape(-1)
    inner = np.tile(inner, L.nnt ** 3)
    return np.repeat(inner, np.asarray(rhoc, np.int64).reshape(-1))


class DeviceImage:
    """An image in device memory (torch tensors), with a spare set of arrays for the drift."""

    def __init__(self, img: Image, device, headroom: float = 1.25, with_pid: bool = True):
        import torch
        self.layout = img.layout
        self.device = device
        self.n_used = img.n_used
        self.n_physical = img.n_particles
        cap = max(int(img.n_used * headroom), 1024)

        def up(a, dtype, shape):
            t = torch.zeros(shape, dtype=dtype, device=device)
            src = torch.from_numpy(np.ascontiguousarray(a))
            t.view(-1)[:src.numel()] = src.reshape(-1).to(device)
            return t
        self.rhoc = up(img.rhoc, torch.int32, (img.rhoc.size,))
        self.idx = up(img.idx_b_r, torch.int64, (img.idx_b_r.size,))
        self.xp = up(img.xp, torch.int16, (cap, 3))
        self.vp = up(img.vp, torch.float32, (cap, 3))
        self.pid = up(img.pid, torch.int64, (cap,)) if with_pid else None
        self._spare = None
        self.cap = cap

    def _alloc_spare(self, cap):
        import torch
        dev = self.device
        self._spare = dict(rhoc=torch.empty_like(self.rhoc), idx=torch.empty_like(self.idx),
                           xp=torch.empty((cap, 3), dtype=torch.int16, device=dev),
                           vp=torch.empty((cap, 3), dtype=torch.float32, device=dev),
                           pid=torch.empty((cap,), dtype=torch.int64, device=dev) if self.pid is not None else None,
                           cap=cap)

    def drift(self, dt_mid: float, vz_max: float, stream=None):
        """drift + buffer_grid + buffer_x + buffer_v of the reference, in one call (the library's
        layout must be configured for this image)."""
        if self._spare is None:
            self._alloc_spare(self.cap)
        n_new, n_phys = ctypes.c_int64(), ctypes.c_int64()
        for attempt in range(2):
            sp = self._spare
            st = lib().cube_drift_device(_dp(self.rhoc), _dp(self.idx), _dp(self.xp), _dp(self.vp),
                                         None if self.pid is None else _dp(self.pid), ctypes.c_int64(self.n_used),
                                         ctypes.c_float(dt_mid), ctypes.c_float(vz_max), _dp(sp["rhoc"]),
                                         _dp(sp["idx"]), _dp(sp["xp"]), _dp(sp["vp"]),
                                         None if sp["pid"] is None else _dp(sp["pid"]), ctypes.c_int64(sp["cap"]),
                                         ctypes.byref(n_new), ctypes.byref(n_phys), _sp(stream))
            if st == CUBE_ERR_CAPACITY and attempt == 0 and n_new.value > sp["cap"]:
                self._alloc_spare(int(n_new.value * 1.25) + 1024)
                continue
            _check(st, "cube_drift_device")
            break
        sp = self._spare
        old = dict(rhoc=self.rhoc, idx=self.idx, xp=self.xp, vp=self.vp, pid=self.pid, cap=self.cap)
        self.rhoc, self.idx, self.xp, self.vp, self.pid, self.cap = (sp["rhoc"], sp["idx"], sp["xp"], sp["vp"],
                                                                     sp["pid"], sp["cap"])
        self._spare = old
        self.n_used = int(n_new.value)
        self.n_physical = int(n_phys.value)

    def buffer_v(self, stream=None):
        """buffer_v: buffer copies take the velocities of the particles they mirror."""
        _check(lib().cube_buffer_v_device(_dp(self.rhoc), _dp(self.idx), _dp(self.vp), ctypes.c_int64(self.n_used),
                                          _sp(stream)), "cube_buffer_v_device")

    def power_spectrum(self, nw: int, nbin: int = 0, stream=None) -> dict:
        """CIC power spectrum of the physical particles (cube_power_spectrum): per linear
        |k| bin (grid units) the mode count, mean |k|, mean |delta_k|^2 / sinc^4 and the
        dimensionless mean 4 pi k^3 |delta_k|^2 / sinc^4."""
        return power_spectrum(self.rhoc, self.idx, self.xp, self.n_used, self.n_physical, nw, nbin, stream)

    def to_host(self) -> Image:
        import torch
        torch.cuda.synchronize()
        L = self.layout
        rhoc = self.rhoc.cpu().numpy().reshape(L.nnt, L.nnt, L.nnt, L.nte, L.nte, L.nte)
        idx = self.idx.cpu().numpy().reshape(L.nnt, L.nnt, L.nnt, L.nte, L.nte)
        n = self.n_used
        pid = self.pid[:n].cpu().numpy() if self.pid is not None else np.zeros(n, np.int64)
        return Image(L, self.xp[:n].cpu().numpy(), self.vp[:n].cpu().numpy(), rhoc, idx, pid,
                     interior_mask(L, rhoc), n_particles=self.n_physical)


def power_spectrum(d_rhoc, d_idx, d_xp, n_used: int, n_physical: int, nw: int, nbin: int = 0, stream=None) -> dict:
    """cube_power_spectrum on device arrays; see DeviceImage.power_spectrum."""
    nb = nbin if nbin > 0 else int(round((nw // 2) * np.sqrt(3.0)))
    bins = np.zeros(4 * (nb + 1), np.float64)
    _check(lib().cube_power_spectrum(_dp(d_rhoc), _dp(d_idx), _dp(d_xp), ctypes.c_int64(n_used),
                                     ctypes.c_int64(n_physical), ctypes.c_int32(nw), ctypes.c_int32(nb), _p(bins),
                                     _sp(stream)), "cube_power_spectrum")
    b = bins.reshape(4, nb + 1)
    modes = b[0]
    with np.errstate(invalid="ignore", divide="ignore"):
        return {"modes": modes, "k": b[1] / modes, "pk": b[2] / modes, "delta2": b[3] / modes}


__all__ = ["DeviceImage", "drift_host", "interior_mask", "power_spectrum", "CubeError"]
