"""ORACLE -- test infrastructure only (see package docstring).

Python drivers for the CPU checkers:

* :class:`RefPP`        the reference's pp_force_kernel.c, compiled per layout
                        (``oracle/_ref``), called through its own C ABI
                        (pp_force_kernel.c:134-141, :393-400);
* :class:`RefCuda`      the reference's CUDA kick (pm3_fft_cuda.cu +
                        pp_force_kernel.cu), compiled per layout for sm_100a,
                        called through its own C ABI (pm3_fft_cuda.cu:516-520,
                        pp_force_kernel.cu:960-963, :515-522);
* :func:`pm3_periodic`  PM3 on one periodic image mesh (restatement of
                        kick.f90:403-568 with wrap-around);
* :func:`pm3_subtile`   PM3 on the reference's per-subtile buffered meshes;
* :func:`green`         Green_3D (Green/Green.f90:1-80) in FP64;
* :func:`ewald`         FP64 Ewald direct summation (physics truth).

The FFT is scipy.fft (pocketfft) in float64 -- a stand-in for FFTW/MKL, whose
result no reference test pins.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
LIB_PATH = os.path.join(HERE, "liboracle.so")
_SRCS = [os.path.join(HERE, "pm3_oracle.c"), os.path.join(HERE, "ewald.c")]

sys.path.insert(0, HERE)
from layouts import GPU_BUILDS, LAYOUTS, ref_gpu_lib_name, ref_lib_name  # noqa: E402

_c_i = ctypes.c_int
_c_i64 = ctypes.c_int64
_c_d = ctypes.c_double
_c_f = ctypes.c_float
_p = ctypes.c_void_p


def build_oracle(force: bool = False) -> str:
    """Compile the C oracle (gcc, OpenMP) into oracle/liboracle.so."""
    if not force and os.path.exists(LIB_PATH):
        if all(os.path.getmtime(LIB_PATH) >= os.path.getmtime(s) for s in _SRCS):
            return LIB_PATH
    subprocess.run(["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", *_SRCS, "-o", LIB_PATH, "-lm"], check=True)
    return LIB_PATH


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH) and os.path.exists(_SRCS[0]):
            build_oracle()
        _LIB = ctypes.CDLL(LIB_PATH)
        _LIB.ewald_forces.restype = None
        _LIB.pm3o_f2max.restype = _c_d
        _LIB.pm3o_f2max_subtile.restype = _c_d
        _LIB.cube_oracle_F_ra64.restype = _c_d
        _LIB.cube_oracle_F_ra64.argtypes = [_c_d, _c_d]
    return _LIB


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_p)


class _OLay(ctypes.Structure):
    _fields_ = [("ng", _c_i), ("nnt", _c_i), ("nns", _c_i), ("ratio_cs", _c_i), ("ngb", _c_i)]


def _olay(layout) -> _OLay:
    return _OLay(layout.ng, layout.nnt, layout.nns, layout.ratio_cs, layout.ngb)


# ----------------------------------------------------------------------------------------------
# reference PP kernel (compiled from the reference's own source)


class RefPP:
    """The reference CPU PP kernel for one compiled layout."""

    def __init__(self, layout, nnest: int = 8, nteam: int = 1):
        p = dict(layout.as_dict())
        p.update(nnest=nnest, nteam=nteam, ncore=nnest * nteam)
        self.layout = layout
        self.path = os.path.join(REF_DIR, ref_lib_name(p))
        if not os.path.exists(self.path):
            raise FileNotFoundError(f"reference build missing: {self.path} (run oracle/build_ref.py)")
        self.lib = ctypes.CDLL(self.path)
        self.lib.c_pp_force_kernel.restype = None
        self.lib.c_pp_force_kernel_tile.restype = None
        self.lib.F_ra.restype = _c_f
        self.lib.F_ra.argtypes = [_c_f, _c_f]
        self.lib.cube_ref_snapshot_size.restype = ctypes.c_size_t
        self.lib.cube_ref_snapshot_copy.restype = ctypes.c_size_t
        self.lib.radix_sort_u32_pair.restype = None

    def F_ra(self, r: float, apm: float) -> float:
        return float(self.lib.F_ra(_c_f(r), _c_f(apm)))

    def kick(self, img, ires_tile, apm3, ratio_sf, mass, a_mid, dt):
        """c_pp_force_kernel (pp_force_kernel.c:393-445) on a copy of img.vp.

        ires_tile[it] is read per parent tile (pp_force_kernel.c:409).
        Returns (vp_new, f2max, vmax[3], ptotal[nnt^3]).
        """
        L = self.layout
        ntile = L.nnt ** 3
        vp = np.ascontiguousarray(img.vp.copy())
        ires = np.zeros(max(L.ns3, ntile), dtype=np.int32)
        ires[:ntile] = np.asarray(ires_tile, dtype=np.int32)
        isort = np.arange(1, L.ns3 + 1, dtype=np.int32)
        ixyz3 = np.zeros((L.ns3, 6), dtype=np.int32)
        apm3 = np.ascontiguousarray(apm3, dtype=np.float32)
        ratio_sf = np.ascontiguousarray(ratio_sf, dtype=np.int32)
        f2 = np.zeros(1, dtype=np.float32)
        vmax = np.zeros(3, dtype=np.float32)
        ptotal = np.zeros(ntile, dtype=np.float64)
        ttotal = np.zeros(ntile, dtype=np.float64)
        self.lib.c_pp_force_kernel(_ptr(isort), _ptr(ires), _ptr(ixyz3), _ptr(apm3), _ptr(ratio_sf),
                                   _ptr(img.rhoc), _ptr(img.idx_b_r), _ptr(img.xp), _ptr(vp),
                                   _c_f(mass), _c_f(a_mid), _c_f(dt), _ptr(f2), _ptr(vmax), _ptr(ptotal),
                                   _ptr(ttotal))
        return vp, float(f2[0]), vmax, ptotal

    def tile(self, img, tile_xyz, iapm, apm3, ratio_sf, mass, a_mid, dt, vp=None, capture=False):
        """c_pp_force_kernel_tile (pp_force_kernel.c:134-391) for one parent tile.

        With capture=True also returns the reference's internal arrays at the
        moment it frees them: keys (sorted), values (sorted original slot),
        cell_start, xf_sorted [3][N], ip_local [N] and af [3][N] (scaled by mass^2).
        """
        L = self.layout
        if vp is None:
            vp = img.vp.copy()
        tile1 = np.array([tile_xyz[0] + 1, tile_xyz[1] + 1, tile_xyz[2] + 1], dtype=np.int32)
        nc1 = np.array([1, 1, 1], dtype=np.int32)
        nc2 = np.array([L.nt] * 3, dtype=np.int32)
        us = np.zeros(3, dtype=np.int32)
        apm3 = np.ascontiguousarray(apm3, dtype=np.float32)
        ratio_sf = np.ascontiguousarray(ratio_sf, dtype=np.int32)
        f2 = np.zeros(1, dtype=np.float32)
        vmax = np.zeros(3, dtype=np.float32)
        ptotal = np.zeros(1, dtype=np.float64)
        ttotal = np.zeros(1, dtype=np.float64)
        if capture:
            self.lib.cube_ref_capture(1)
        self.lib.c_pp_force_kernel_tile(_c_i(0), _c_i(iapm), _ptr(tile1), _ptr(nc1), _ptr(nc2), _ptr(us),
                                        _ptr(ratio_sf), _ptr(apm3), _ptr(img.rhoc), _ptr(img.idx_b_r),
                                        _ptr(img.xp), _ptr(vp), _c_f(mass), _c_f(a_mid), _c_f(dt), _ptr(f2),
                                        _ptr(vmax), _ptr(ptotal), _ptr(ttotal))
        out = dict(vp=vp, f2max=float(f2[0]), vmax=vmax, ncount=int(ptotal[0]), seconds=float(ttotal[0]))
        if capture:
            def snap(slot, dtype):
                n = int(self.lib.cube_ref_snapshot_size(_c_i(slot)))
                buf = np.empty(n // np.dtype(dtype).itemsize, dtype=dtype)
                self.lib.cube_ref_snapshot_copy(_c_i(slot), _ptr(buf), ctypes.c_size_t(n))
                return buf
            ip_local = snap(3, np.int64)
            N = ip_local.shape[0]
            out.update(keys=snap(4, np.uint32)[:N], values=snap(5, np.uint32)[:N],
                       cell_start=snap(9, np.int32), xf_sorted=snap(8, np.float32).reshape(3, N),
                       ip_local=ip_local, af=snap(2, np.float32).reshape(3, N))
            self.lib.cube_ref_capture(0)
        return out

    def radix_sort(self, keys, vals):
        k = np.ascontiguousarray(keys, dtype=np.uint32).copy()
        v = np.ascontiguousarray(vals, dtype=np.uint32).copy()
        self.lib.radix_sort_u32_pair(_ptr(k), _ptr(v), _c_i(k.shape[0]))
        return k, v


class RefCuda:
    """The reference's CUDA kick for one compiled layout (``GPU_BUILDS``).

    PM3 (pm3_fft_cuda.cu:516-620) leaves its velocity change in the reference's
    shared device accumulator; :meth:`kick` reads it there through
    ``c_gpu_velocity_get`` (pp_force_kernel.cu:515-522), then runs the reference
    PP (pp_force_kernel.cu:960-1050), which adds its own change and merges both
    into the host velocities.

    The reference ends the process (``exit``/``abort``) on any capacity or
    metadata error, so every input is checked here first against the limits the
    reference would enforce (pp_force_kernel.cu:45-51, :818-821, :964-1000,
    pm3_fft_cuda.cu:392-401).
    """

    _cudart = None

    def __init__(self, name: str):
        self.params = dict(GPU_BUILDS[name])
        self.path = os.path.join(REF_DIR, ref_gpu_lib_name(self.params))
        if not os.path.exists(self.path):
            raise FileNotFoundError(f"reference CUDA build missing: {self.path} (run oracle/build_ref.py)")
        self.lib = ctypes.CDLL(self.path)
        for f in ("c_pm3_force_kernel", "c_pp_force_kernel", "c_gpu_velocity_finalize", "c_pm3_fft_finalize"):
            getattr(self.lib, f).restype = None
        self.lib.c_gpu_velocity_get.restype = ctypes.c_void_p
        self.lib.c_gpu_velocity_get.argtypes = [_c_i]
        if RefCuda._cudart is None:
            home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
            RefCuda._cudart = ctypes.CDLL(os.path.join(home, "lib64", "libcudart.so.12"))
            RefCuda._cudart.cudaMemcpy.restype = _c_i
            RefCuda._cudart.cudaMemcpy.argtypes = [_p, _p, ctypes.c_size_t, _c_i]
        p = self.params
        nc = p["ng"] // p["ratio_cs"]
        nt = nc // p["nnt"]
        nte = nt + 2 * (p["ngb"] // p["ratio_cs"])
        np_image = (nc * p["np_nc"]) ** 3
        a = nte * 1.0 / nt
        # the reference's own capacity arithmetic, in its order of operations (pp_force_kernel.cu:45-51)
        self.np_image_max = int(np_image * a * a * a * p["image_buffer"])
        self.np_tile_max = int(np_image // p["nnt"] ** 3 * (a * a * a) * p["tile_buffer"])

    def _check(self, img, ires, ixyz3):
        L = img.layout
        p = self.params
        for k in ("ng", "nnt", "nns", "ratio_cs", "ngb"):
            if getattr(L, k) != p[k]:
                raise ValueError(f"image layout {k}={getattr(L, k)} differs from the build's {p[k]}")
        if p["ng"] > 512 or L.nt + 2 >= 128:
            raise ValueError("layout outside the reference CUDA PP's exact range")
        if not (0 <= img.n_used <= min(self.np_image_max, 2 ** 31 - 1)):
            raise ValueError(f"{img.n_used} stored particles exceed the reference capacity {self.np_image_max}")
        ires = np.asarray(ires)
        if ires.min() < 2 or ires.max() > 6:
            raise ValueError("ires outside 2..6")
        ix = np.asarray(ixyz3)
        if ix[:, :3].min() < 1 or ix[:, :3].max() > L.nns or ix[:, 3:].min() < 1 or ix[:, 3:].max() > L.nnt:
            raise ValueError("ixyz3 outside the layout")
        # particles staged per parent tile: the subtile cells plus a one coarse-cell ring
        ncb = L.ncb
        r = img.rhoc.reshape(L.nnt ** 3, L.nte, L.nte, L.nte)[:, ncb - 1:ncb + L.nt + 1, ncb - 1:ncb + L.nt + 1,
                                                               ncb - 1:ncb + L.nt + 1]
        if int(r.reshape(L.nnt ** 3, -1).sum(axis=1).max()) > self.np_tile_max:
            raise ValueError("a parent tile exceeds the reference capacity np_tile_max")

    def _d2h(self, dptr: int, n: int) -> np.ndarray:
        out = np.empty(n, dtype=np.float32)
        st = RefCuda._cudart.cudaMemcpy(out.ctypes.data, dptr, n * 4, 2)
        if st != 0:
            raise RuntimeError(f"cudaMemcpy of the reference accumulator failed ({st})")
        return out

    def kick(self, img, isort, ires, ixyz3, apm3, ratio_sf, greens: dict, mass, a_mid, dt, vp=None):
        """PM3 then PP through the reference's CUDA path, as kick.f90:143-205 calls them.

        Returns dict(dv_pm3 float32 [n_used,3] (the PM3 change alone), f2max_pm3,
        ptotal_pm3 [ns3], vp (after both), f2max_pp, vmax [3], ptotal_pp [ns3]).
        """
        L = img.layout
        isort = np.ascontiguousarray(isort, dtype=np.int32)
        ires = np.ascontiguousarray(ires, dtype=np.int32)
        ixyz3 = np.ascontiguousarray(ixyz3, dtype=np.int32)
        apm3 = np.ascontiguousarray(apm3, dtype=np.float32)
        ratio_sf = np.ascontiguousarray(ratio_sf, dtype=np.int32)
        self._check(img, ires, ixyz3)
        # one FFT batch per (parent tile, level) holds at most 64 subtiles (pm3_fft_cuda.cu:392-401)
        if L.nns ** 3 > 64:
            raise ValueError("more than 64 subtiles per parent tile")
        gk = []
        keep = []
        for lev in range(2, 7):
            g = greens.get(lev) if greens else None
            if g is not None:
                g = np.ascontiguousarray(g, dtype=np.float32)
                keep.append(g)
                gk.append(g.ctypes.data_as(_p))
            else:
                gk.append(None)
        used = set(int(v) for v in ires.tolist())
        for lev in used:
            rsf = int(ratio_sf[lev - 1])
            n = L.ntt * L.ratio_cs * rsf + 2 * L.ratio_cs * rsf
            g = greens.get(lev)
            if g is None or g.size != n * n * (n // 2 + 1):
                raise ValueError(f"level {lev} needs a Green table of {n}^2 x {n // 2 + 1}")
        vp = np.ascontiguousarray(img.vp.copy() if vp is None else vp, dtype=np.float32)
        f2 = np.zeros(1, np.float32)
        vm = np.zeros(3, np.float32)
        pt = np.zeros(L.ns3, np.float64)
        self.lib.c_pm3_force_kernel(_ptr(isort), _ptr(ires), _ptr(ixyz3), _ptr(ratio_sf), _ptr(img.rhoc),
                                    _ptr(img.idx_b_r), _ptr(img.xp), *gk, _ptr(vp), _c_f(mass), _c_f(a_mid),
                                    _c_f(dt), _ptr(f2), _ptr(vm), _ptr(pt))
        n_used = img.n_used
        dv = self._d2h(self.lib.c_gpu_velocity_get(_c_i(n_used)), 3 * n_used).reshape(n_used, 3)
        out = dict(dv_pm3=dv, f2max_pm3=float(f2[0]), ptotal_pm3=pt.copy())
        f2p = np.zeros(1, np.float32)
        vmax = np.zeros(3, np.float32)
        ptp = np.zeros(L.ns3, np.float64)
        tt = np.zeros(L.ns3, np.float64)
        self.lib.c_pp_force_kernel(_ptr(isort), _ptr(ires), _ptr(ixyz3), _ptr(apm3), _ptr(ratio_sf),
                                   _ptr(img.rhoc), _ptr(img.idx_b_r), _ptr(img.xp), _ptr(vp), _c_f(mass),
                                   _c_f(a_mid), _c_f(dt), _ptr(f2p), _ptr(vmax), _ptr(ptp), _ptr(tt))
        del keep
        out.update(vp=vp, f2max_pp=float(f2p[0]), vmax=vmax, ptotal_pp=ptp, seconds_pp=tt)
        return out

    def kick_wall(self, img, isort, ires, ixyz3, apm3, ratio_sf, greens: dict, mass, a_mid, dt, vp):
        """The two entry points as kick.f90:143-205 calls them (PM3, then PP, which applies the
        PM3 change from the device accumulator), on the caller's host arrays; vp is kicked in
        place.  Returns (seconds of c_pm3_force_kernel, seconds of c_pp_force_kernel), wall clock
        around each call (each returns with its results on the host)."""
        import time
        L = img.layout
        isort = np.ascontiguousarray(isort, dtype=np.int32)
        ires = np.ascontiguousarray(ires, dtype=np.int32)
        ixyz3 = np.ascontiguousarray(ixyz3, dtype=np.int32)
        apm3 = np.ascontiguousarray(apm3, dtype=np.float32)
        ratio_sf = np.ascontiguousarray(ratio_sf, dtype=np.int32)
        self._check(img, ires, ixyz3)
        if L.nns ** 3 > 64:
            raise ValueError("more than 64 subtiles per parent tile")
        if vp.dtype != np.float32 or not vp.flags.c_contiguous or vp.shape != img.vp.shape:
            raise ValueError("vp must be a C-contiguous float32 array shaped like img.vp")
        keep = [np.ascontiguousarray(greens[lev], dtype=np.float32) if greens.get(lev) is not None else None
                for lev in range(2, 7)]
        for lev in set(int(v) for v in ires.tolist()):
            n = L.ntt * L.ratio_cs * int(ratio_sf[lev - 1]) + 2 * L.ratio_cs * int(ratio_sf[lev - 1])
            if keep[lev - 2] is None or keep[lev - 2].size != n * n * (n // 2 + 1):
                raise ValueError(f"level {lev} needs a Green table of {n}^2 x {n // 2 + 1}")
        gk = [None if g is None else g.ctypes.data_as(_p) for g in keep]
        f2 = np.zeros(1, np.float32)
        vm = np.zeros(3, np.float32)
        pt = np.zeros(L.ns3, np.float64)
        tt = np.zeros(L.ns3, np.float64)
        t0 = time.perf_counter()
        self.lib.c_pm3_force_kernel(_ptr(isort), _ptr(ires), _ptr(ixyz3), _ptr(ratio_sf), _ptr(img.rhoc),
                                    _ptr(img.idx_b_r), _ptr(img.xp), *gk, _ptr(vp), _c_f(mass), _c_f(a_mid),
                                    _c_f(dt), _ptr(f2), _ptr(vm), _ptr(pt))
        t1 = time.perf_counter()
        self.lib.c_pp_force_kernel(_ptr(isort), _ptr(ires), _ptr(ixyz3), _ptr(apm3), _ptr(ratio_sf),
                                   _ptr(img.rhoc), _ptr(img.idx_b_r), _ptr(img.xp), _ptr(vp), _c_f(mass),
                                   _c_f(a_mid), _c_f(dt), _ptr(f2), _ptr(vm), _ptr(pt), _ptr(tt))
        t2 = time.perf_counter()
        del keep
        return t1 - t0, t2 - t1

    def finalize(self):
        self.lib.c_gpu_velocity_finalize()
        self.lib.c_pm3_fft_finalize()


def ref_layout_params(name: str) -> dict:
    return dict(LAYOUTS[name])


# ----------------------------------------------------------------------------------------------
# PM3 restatement


def _fft_workers() -> int:
    return max(1, os.cpu_count() or 1)


def green(n: int, apm_soft: float, apm_range: float, gridsize: float, p_order: int = 2) -> np.ndarray:
    """Green_3D (Green.f90:1-80) -> float32 [n][n][n/2+1]."""
    G = np.empty((n, n, n // 2 + 1), dtype=np.float32)
    lib().pm3o_green(_c_i64(n), _c_d(apm_soft), _c_d(apm_range), _c_d(gridsize), _c_i(p_order), _ptr(G))
    return G


def green_mirrored(n: int, apm_soft: float, apm_range: float, gridsize: float, p_order: int = 2) -> np.ndarray:
    """:func:`green` from a quarter of the work (rows mirrored along the second and third axes);
    equal to it up to the last bit of the FP64 alias sums (far below its float rounding)."""
    G = np.empty((n, n, n // 2 + 1), dtype=np.float32)
    lib().pm3o_green_mirrored(_c_i64(n), _c_d(apm_soft), _c_d(apm_range), _c_d(gridsize), _c_i(p_order), _ptr(G))
    return G


def _solve(rho: np.ndarray, G: np.ndarray) -> np.ndarray:
    import scipy.fft as sf
    n = rho.shape[0]
    rhok = sf.rfftn(rho, workers=_fft_workers())
    rhok *= G
    return sf.irfftn(rhok, s=(n, n, n), workers=_fft_workers())


def pm3_periodic(img, rsf: int, G: np.ndarray, mass: float, a_mid: float, dt: float, fft_dtype=np.float64):
    """PM3 on one periodic image mesh n = ng*rsf.  Returns dict(vp, f2max, vmax, dv, force)."""
    L = img.layout
    n = L.ng * rsf
    ol = _olay(L)
    rho = np.empty((n, n, n), dtype=np.float64)
    lib().pm3o_deposit_periodic(ctypes.byref(ol), _ptr(img.xp), _ptr(img.rhoc), _ptr(img.idx_b_r), _c_i(rsf),
                                _ptr(rho))
    rho *= mass  # kick.f90:463
    phi = _solve(rho.astype(fft_dtype), G).astype(np.float64)
    del rho
    force = np.empty((3, n, n, n), dtype=np.float64)
    lib().pm3o_force_periodic(_c_i64(n), _ptr(phi), _c_d(float(n) ** 3), _ptr(force))
    del phi
    f2max = float(lib().pm3o_f2max(_c_i64(n ** 3), _ptr(force)))
    vp = img.vp.copy()
    dv = np.zeros((img.n_used, 3), dtype=np.float64)
    vmax = np.zeros(3, dtype=np.float32)
    kick = float(np.float32(a_mid) * np.float32(dt) / np.float32(6.0)) / np.pi
    lib().pm3o_gather_periodic(ctypes.byref(ol), _ptr(img.xp), _ptr(img.rhoc), _ptr(img.idx_b_r), _c_i(rsf),
                               _ptr(force), _c_d(kick), _ptr(vp), _ptr(dv), _ptr(vmax))
    return dict(vp=vp, f2max=f2max, vmax=vmax, dv=dv, force=force)


def pm3_subtile(img, ires, ixyz3, ratio_sf, greens: dict, mass: float, a_mid: float, dt: float):
    """PM3 on the reference's per-subtile buffered meshes (kick.f90:149-178).

    greens maps level (2..6) -> Green table of that level's mesh (nft^3 half spectrum).
    Returns dict(vp, f2max, vmax, dv).
    """
    L = img.layout
    ol = _olay(L)
    ixyz3 = np.ascontiguousarray(ixyz3, dtype=np.int32)
    vp = img.vp.copy()
    dv = np.zeros((img.n_used, 3), dtype=np.float64)
    f2max = 0.0
    vmax = np.zeros(3, dtype=np.float32)
    kick = float(np.float32(a_mid) * np.float32(dt) / np.float32(6.0)) / np.pi
    for it in range(L.ns3):
        lev = int(ires[it])
        rsf = int(ratio_sf[lev - 1])
        nfp = L.ntt * L.ratio_cs * rsf
        nfb = L.ratio_cs * rsf
        nft = nfp + 2 * nfb
        rho = np.empty((nft, nft, nft), dtype=np.float64)
        lib().pm3o_deposit_subtile(ctypes.byref(ol), _ptr(img.xp), _ptr(img.rhoc), _ptr(img.idx_b_r), _ptr(ixyz3),
                                   _c_i(it), _c_i(rsf), _ptr(rho))
        rho *= mass
        phi = _solve(rho, greens[lev])
        force = np.empty((3, nft, nft, nft), dtype=np.float64)
        lib().pm3o_force_periodic(_c_i64(nft), _ptr(phi), _c_d(float(nft) ** 3), _ptr(force))
        f2max = max(f2max, float(lib().pm3o_f2max_subtile(_c_i64(nft), _c_i64(nfp), _c_i64(nfb), _ptr(force))))
        vm = np.zeros(3, dtype=np.float32)
        lib().pm3o_gather_subtile(ctypes.byref(ol), _ptr(img.xp), _ptr(img.rhoc), _ptr(img.idx_b_r), _ptr(ixyz3),
                                  _c_i(it), _c_i(rsf), _ptr(force), _c_d(kick), _ptr(vp), _ptr(dv), _ptr(vm))
        vmax = np.maximum(vmax, vm)
    return dict(vp=vp, f2max=f2max, vmax=vmax, dv=dv)


def pm1(img, apm1c: float, mass: float, a_mid: float, dt: float):
    """PM1 (particle_mesh.f90, pm_layer 1) on the periodic coarse mesh nc^3 with
    Green_3D(nc, apm1c, 0, ratio_cs).  Returns dict(vp, f2max, vmax, dv)."""
    L = img.layout
    n = L.nc
    ol = _olay(L)
    G = green(n, apm1c, 0.0, float(L.ratio_cs))
    rho = np.empty((n, n, n), dtype=np.float64)
    lib().pm1o_deposit(ctypes.byref(ol), _ptr(img.xp), _ptr(img.rhoc), _ptr(img.idx_b_r), _ptr(rho))
    rho *= mass
    phi = _solve(rho, G)
    force = np.empty((3, n, n, n), dtype=np.float64)
    lib().pm3o_force_periodic(_c_i64(n), _ptr(phi), _c_d(float(n) ** 3), _ptr(force))
    f2max = float(lib().pm3o_f2max(_c_i64(n ** 3), _ptr(force)))
    vp = img.vp.copy()
    dv = np.zeros((img.n_used, 3), dtype=np.float64)
    vmax = np.zeros(3, dtype=np.float32)
    kick = float(np.float32(a_mid) * np.float32(dt) / np.float32(6.0)) / np.pi
    lib().pm1o_gather(ctypes.byref(ol), _ptr(img.xp), _ptr(img.rhoc), _ptr(img.idx_b_r), _ptr(force), _c_d(kick),
                      _ptr(vp), _ptr(dv), _ptr(vmax))
    return dict(vp=vp, f2max=f2max, vmax=vmax, dv=dv)


def pm2(img, apm2: float, apm1: float, mass: float, a_mid: float, dt: float):
    """PM2 (pm_thread with the parameters of kick.f90:82-88) on every tile's buffered fine mesh,
    ngt = (nt + 2 ncb) ratio_cs, with Green_3D(ngt, apm2, apm1, 1).  Returns dict(vp, f2max, vmax, dv)."""
    L = img.layout
    nft = L.nte * L.ratio_cs
    nfp, nfb = L.nt * L.ratio_cs, L.ncb * L.ratio_cs
    ol = _olay(L)
    G = green(nft, apm2, apm1, 1.0)
    vp = img.vp.copy()
    dv = np.zeros((img.n_used, 3), dtype=np.float64)
    f2max = 0.0
    vmax = np.zeros(3, dtype=np.float32)
    kick = float(np.float32(a_mid) * np.float32(dt) / np.float32(6.0)) / np.pi
    for t in range(L.nnt ** 3):
        rho = np.empty((nft, nft, nft), dtype=np.float64)
        lib().pm2o_deposit(ctypes.byref(ol), _ptr(img.xp), _ptr(img.rhoc), _ptr(img.idx_b_r), _c_i(t), _ptr(rho))
        rho *= mass
        phi = _solve(rho, G)
        force = np.empty((3, nft, nft, nft), dtype=np.float64)
        lib().pm3o_force_periodic(_c_i64(nft), _ptr(phi), _c_d(float(nft) ** 3), _ptr(force))
        f2max = max(f2max, float(lib().pm3o_f2max_subtile(_c_i64(nft), _c_i64(nfp), _c_i64(nfb), _ptr(force))))
        vm = np.zeros(3, dtype=np.float32)
        lib().pm2o_gather(ctypes.byref(ol), _ptr(img.xp), _ptr(img.rhoc), _ptr(img.idx_b_r), _c_i(t), _ptr(force),
                          _c_d(kick), _ptr(vp), _ptr(dv), _ptr(vm))
        vmax = np.maximum(vmax, vm)
    return dict(vp=vp, f2max=f2max, vmax=vmax, dv=dv)


# ----------------------------------------------------------------------------------------------
# FP64 truth


def ewald(pos: np.ndarray, L: float, app: float, targets: np.ndarray, alpha: float | None = None,
          tol: float = 1e-9):
    """FP64 periodic softened force on the target particles (see ewald.c).

    pos: float64 [N,3] fine-cell positions of each physical particle once.
    """
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    targets = np.ascontiguousarray(targets, dtype=np.int64)
    rcut = 0.5 * L
    if alpha is None:
        # erfc(alpha rcut) ~ tol  ->  alpha rcut ~ sqrt(-ln tol)
        alpha = np.sqrt(-np.log(tol)) / rcut
    kmax = 2.0 * alpha * np.sqrt(-np.log(tol))
    nmax = int(np.ceil(kmax * L / (2 * np.pi)))
    F = np.zeros((targets.shape[0], 3), dtype=np.float64)
    lib().ewald_forces(_c_i64(pos.shape[0]), _ptr(pos), _c_d(L), _c_d(app), _c_i64(targets.shape[0]),
                       _ptr(targets), _c_d(alpha), _c_d(rcut), _c_i(nmax), _ptr(F))
    return F


def F_ra64(r: float, apm: float) -> float:
    return float(lib().cube_oracle_F_ra64(r, apm))
