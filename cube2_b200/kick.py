"""Python mirror of the reference's fine-scale kick interface.

``FineKick`` binds the C-ABI of ``libcube2_b200.so`` (include/cube2_b200.h)
with numpy arrays in the reference's layout (see ``layout.py``).  The methods
keep the reference names and argument meanings:

* :meth:`FineKick.c_pm3_force_kernel` -- kick.f90:31-45 / pm3_fft_cuda.cu:516
* :meth:`FineKick.c_pp_force_kernel`  -- kick.f90:13-30 / pp_force_kernel.cu:960
* :meth:`FineKick.kick_fine`          -- both in one call
* :meth:`FineKick.kick_fine_device`   -- the same on device-resident (torch) arrays

There is no CPU path: if the shared library is missing or no GPU is visible,
every call raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .layout import Image, Layout

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcube2_b200.so")

CUBE_PM3_SUBTILE = 0
CUBE_PM3_PERIODIC = 1
CUBE_PM3_TILE_PERIODIC = 2

_STATUS = {0: "ok", 1: "invalid argument or subtile metadata", 2: "layout not configured", 3: "CUDA runtime error",
           4: "cuFFT error", 5: "device capacity check failed", 6: "no CUDA device visible",
           7: "bounded device wait timed out"}


class CubeError(RuntimeError):
    def __init__(self, status: int, where: str):
        super().__init__(f"{where}: status {status} ({_STATUS.get(status, 'unknown')})")
        self.status = status


class CLayout(ctypes.Structure):
    _fields_ = [("ng", ctypes.c_int32), ("nnt", ctypes.c_int32), ("nns", ctypes.c_int32),
                ("ratio_cs", ctypes.c_int32), ("ngb", ctypes.c_int32), ("app", ctypes.c_float),
                ("pm3_mode", ctypes.c_int32), ("apm3f", ctypes.c_float), ("apm_range", ctypes.c_float),
                ("p_order", ctypes.c_int32)]


_LIB = None

# every symbol include/cube2_b200.h declares
EXPORTS = ("cube_set_layout", "cube_get_layout", "cube_last_error", "cube_error_string", "c_pm3_force_kernel",
           "c_pp_force_kernel", "c_pm3_fft_finalize", "c_gpu_velocity_finalize", "cube_pm3_force", "cube_pp_force",
           "cube_kick_fine", "cube_kick_fine_device", "cube_pp_bin_tile", "cube_pp_pair_count", "cube_green_table",
           "cube_force_truth_fp64", "cube_stage_times", "cube_enable_timing", "cube_timing_read",
           "cube_launch_count", "cube_fp32_peak_probe", "cube_pp_force_noalloc", "cube_kick_graph_create",
           "cube_kick_graph_launch", "cube_kick_graph_destroy", "cube_mlp_create", "cube_mlp_destroy",
           "cube_mlp_get_params", "cube_mlp_features", "cube_mlp_train_step", "cube_mlp_forward", "cube_mlp_kick",
           "cube_pp_set_shape", "cube_pp_shapes", "cube_drift_device", "cube_drift", "cube_buffer_v_device",
           "cube_power_spectrum", "cube_snapshot_write", "cube_snapshot_read", "cube_pm1_force_device",
           "cube_pm2_force_device", "cube_pp_work_stats", "cube_kick_sums", "cube_learned_fallback")


def lib() -> ctypes.CDLL:
    """Load the shared library (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing: run `python -m cube2_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name in EXPORTS:
            getattr(L, name)
        L.cube_error_string.restype = ctypes.c_char_p
        L.c_pm3_force_kernel.restype = None
        L.c_pp_force_kernel.restype = None
        L.c_pm3_fft_finalize.restype = None
        L.c_gpu_velocity_finalize.restype = None
        _LIB = L
    return _LIB


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.c_void_p)


def _check(status: int, where: str):
    if status != 0:
        raise CubeError(status, where)


def _c32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class CPPShape(ctypes.Structure):
    _fields_ = [("chunk", ctypes.c_int32), ("jtile", ctypes.c_int32), ("unroll", ctypes.c_int32),
                ("blocks", ctypes.c_int32), ("packed", ctypes.c_int32), ("ms", ctypes.c_float)]


def pp_set_shape(shape: int = -1):
    """Use PP kernel shape `shape` for every PP kick, or autotune (-1, the default)."""
    _check(lib().cube_pp_set_shape(ctypes.c_int32(shape)), "cube_pp_set_shape")


def pp_shapes():
    """(table, current): the PP kernel shapes as dicts (chunk, jtile, unroll, blocks, packed, ms of
    the last tuning or -1) and the index of the shape the last PP kick used."""
    n, cur = ctypes.c_int32(), ctypes.c_int32()
    _check(lib().cube_pp_shapes(None, 0, ctypes.byref(n), ctypes.byref(cur)), "cube_pp_shapes")
    arr = (CPPShape * n.value)()
    _check(lib().cube_pp_shapes(arr, n.value, None, None), "cube_pp_shapes")
    table = [{k: getattr(e, k) for k, _ in CPPShape._fields_} for e in arr]
    return table, cur.value


def kick_sums(d_rhoc, d_idx, n_used, d_va, d_vb, mass=1.0, stream=None) -> dict:
    """FP64 momentum and kinetic-energy change of the physical particles between two device
    velocity arrays (torch tensors or device pointers) of one image (cube_kick_sums)."""
    def dp(x):
        return ctypes.c_void_p(x if isinstance(x, int) else x.data_ptr())
    out = np.zeros(8, np.float64)
    s = None if stream is None else ctypes.c_void_p(stream if isinstance(stream, int) else stream.cuda_stream)
    _check(lib().cube_kick_sums(dp(d_rhoc), dp(d_idx), ctypes.c_int64(int(n_used)), dp(d_va), dp(d_vb),
                                ctypes.c_float(mass), _p(out), s), "cube_kick_sums")
    return dict(momentum=out[0:3].copy(), kinetic_energy=float(out[3]), momentum_scale=out[4:7].copy(),
                particles=int(out[7]))


def pp_work_stats() -> dict:
    """The PP work list of the last PP kick: items, items of split cells, grouped items, largest item."""
    out = np.zeros(4, np.int64)
    _check(lib().cube_pp_work_stats(_p(out)), "cube_pp_work_stats")
    return dict(items=int(out[0]), split_items=int(out[1]), grouped_items=int(out[2]), max_ni=int(out[3]))


class KickGraph:
    """A captured device kick; ``launch(stream)`` replays it, ``close()`` frees it."""

    def __init__(self, handle: ctypes.c_void_p):
        self.handle = handle

    def launch(self, stream=None):
        s = None if stream is None else ctypes.c_void_p(stream if isinstance(stream, int) else stream.cuda_stream)
        _check(lib().cube_kick_graph_launch(self.handle, s), "cube_kick_graph_launch")

    def close(self):
        if self.handle:
            lib().cube_kick_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FineKick:
    """Fine-scale kick (PM3 + PP) on the GPU for one layout."""

    def __init__(self, layout: Layout, pm3_mode: int = CUBE_PM3_PERIODIC, apm3f: float = 4.0,
                 apm_range: float = 0.0):
        self.layout = layout
        self.pm3_mode = pm3_mode
        self.apm3f = apm3f
        self.apm_range = apm_range
        self.configure()

    def configure(self):
        L = self.layout
        cl = CLayout(L.ng, L.nnt, L.nns, L.ratio_cs, L.ngb, L.app, self.pm3_mode, self.apm3f, self.apm_range, 2)
        _check(lib().cube_set_layout(ctypes.byref(cl)), "cube_set_layout")

    @staticmethod
    def _gk(greens):
        arr = (ctypes.c_void_p * 5)()
        keep = []
        if greens:
            for lev in range(2, 7):
                g = greens.get(lev)
                if g is not None:
                    g = _f32(g)
                    keep.append(g)
                    arr[lev - 2] = g.ctypes.data
        return arr, keep

    # -- reference entry points ------------------------------------------------------------------
    def c_pm3_force_kernel(self, img: Image, isort, ires, ixyz3, ratio_sf, mass, a_mid, dt, greens=None,
                           vp=None):
        """PM3 kick; returns (vp, f2max, vmax[3], ptotal[ns3]). vp is updated in place if given."""
        L = self.layout
        vp = img.vp.copy() if vp is None else vp
        f2 = np.zeros(1, np.float32)
        vmax = np.zeros(3, np.float32)
        pt = np.zeros(L.ns3, np.float64)
        gk, keep = self._gk(greens)
        isort, ires, ixyz3, ratio_sf = _c32(isort), _c32(ires), _c32(ixyz3), _c32(ratio_sf)
        st = lib().cube_pm3_force(_p(isort), _p(ires), _p(ixyz3), _p(ratio_sf), _p(img.rhoc), _p(img.idx_b_r),
                                  _p(img.xp), gk, _p(vp), ctypes.c_float(mass), ctypes.c_float(a_mid),
                                  ctypes.c_float(dt), _p(f2), _p(vmax), _p(pt))
        _check(st, "c_pm3_force_kernel")
        del keep
        return vp, float(f2[0]), vmax, pt

    def c_pp_force_kernel(self, img: Image, isort, ires, ixyz3, apm3, ratio_sf, mass, a_mid, dt, vp=None):
        """PP kick; returns (vp, f2max, vmax[3], ptotal[ns3], ttotal[ns3])."""
        L = self.layout
        vp = img.vp.copy() if vp is None else vp
        f2 = np.zeros(1, np.float32)
        vmax = np.zeros(3, np.float32)
        pt = np.zeros(L.ns3, np.float64)
        tt = np.zeros(L.ns3, np.float64)
        isort, ires, ixyz3, ratio_sf, apm3 = _c32(isort), _c32(ires), _c32(ixyz3), _c32(ratio_sf), _f32(apm3)
        st = lib().cube_pp_force(_p(isort), _p(ires), _p(ixyz3), _p(apm3), _p(ratio_sf), _p(img.rhoc),
                                 _p(img.idx_b_r), _p(img.xp), _p(vp), ctypes.c_float(mass), ctypes.c_float(a_mid),
                                 ctypes.c_float(dt), _p(f2), _p(vmax), _p(pt), _p(tt))
        _check(st, "c_pp_force_kernel")
        return vp, float(f2[0]), vmax, pt, tt

    def kick_fine(self, img: Image, isort, ires, ixyz3, apm3, ratio_sf, mass, a_mid, dt, greens=None, vp=None):
        """PM3 + PP; returns (vp, out[5] = f2max_pm3, f2max_pp, vmax xyz)."""
        vp = img.vp.copy() if vp is None else vp
        out = np.zeros(5, np.float32)
        gk, keep = self._gk(greens)
        isort, ires, ixyz3, ratio_sf, apm3 = _c32(isort), _c32(ires), _c32(ixyz3), _c32(ratio_sf), _f32(apm3)
        st = lib().cube_kick_fine(_p(isort), _p(ires), _p(ixyz3), _p(apm3), _p(ratio_sf), _p(img.rhoc),
                                  _p(img.idx_b_r), _p(img.xp), gk, _p(vp), ctypes.c_float(mass),
                                  ctypes.c_float(a_mid), ctypes.c_float(dt), _p(out), None)
        _check(st, "cube_kick_fine")
        del keep
        return vp, out

    def kick_fine_device(self, d_rhoc, d_idx, d_xp, n_used, d_vp, d_out, isort, ires, ixyz3, apm3, ratio_sf,
                         mass, a_mid, dt, stream=None, greens=None):
        """Enqueue the kick on device arrays (torch tensors or raw device pointers as int)."""
        def dp(x):
            return ctypes.c_void_p(x if isinstance(x, int) else x.data_ptr())
        gk, keep = self._gk(greens)
        isort, ires, ixyz3, ratio_sf, apm3 = _c32(isort), _c32(ires), _c32(ixyz3), _c32(ratio_sf), _f32(apm3)
        s = None if stream is None else ctypes.c_void_p(stream if isinstance(stream, int) else stream.cuda_stream)
        st = lib().cube_kick_fine_device(_p(isort), _p(ires), _p(ixyz3), _p(apm3), _p(ratio_sf), dp(d_rhoc),
                                         dp(d_idx), dp(d_xp), ctypes.c_int64(int(n_used)), gk, dp(d_vp),
                                         ctypes.c_float(mass), ctypes.c_float(a_mid), ctypes.c_float(dt), dp(d_out),
                                         s)
        _check(st, "cube_kick_fine_device")
        del keep

    def kick_graph(self, d_rhoc, d_idx, d_xp, n_used, d_vp, d_out, isort, ires, ixyz3, apm3, ratio_sf, mass,
                   a_mid, dt) -> "KickGraph":
        """Capture the device kick on these arrays as a CUDA graph (cube_kick_graph_create)."""
        def dp(x):
            return ctypes.c_void_p(x if isinstance(x, int) else x.data_ptr())
        isort, ires, ixyz3, ratio_sf, apm3 = _c32(isort), _c32(ires), _c32(ixyz3), _c32(ratio_sf), _f32(apm3)
        h = ctypes.c_void_p()
        st = lib().cube_kick_graph_create(_p(isort), _p(ires), _p(ixyz3), _p(apm3), _p(ratio_sf), dp(d_rhoc),
                                          dp(d_idx), dp(d_xp), ctypes.c_int64(int(n_used)), dp(d_vp),
                                          ctypes.c_float(mass), ctypes.c_float(a_mid), ctypes.c_float(dt), dp(d_out),
                                          ctypes.byref(h))
        _check(st, "cube_kick_graph_create")
        return KickGraph(h)

    # -- inspection ------------------------------------------------------------------------------
    def pp_bin_tile(self, img: Image, tile: int, ires, ixyz3, ratio_sf, spatial: bool = False):
        """Binning of one parent tile: dict(keys, ip, cell_start, xf[3][N]).

        spatial=False: the reference's order inside each PP cell; True: the kick's order."""
        L = self.layout
        rcp = int(max(np.asarray(ratio_sf)[np.asarray(ires) - 1]))
        S = rcp * (L.nt + 2)
        grid = S ** 3
        cap = img.n_used
        keys = np.zeros(max(cap, 1), np.uint32)
        ip = np.zeros(max(cap, 1), np.int64)
        cs = np.zeros(grid + 1, np.int32)
        xf = np.zeros(3 * max(cap, 1), np.float32)
        n_out = np.zeros(1, np.int64)
        g_out = np.zeros(1, np.int64)
        ires, ixyz3, ratio_sf = _c32(ires), _c32(ixyz3), _c32(ratio_sf)
        st = lib().cube_pp_bin_tile(_p(ires), _p(ixyz3), _p(ratio_sf), _p(img.rhoc), _p(img.idx_b_r), _p(img.xp),
                                    ctypes.c_int32(tile), ctypes.c_int32(1 if spatial else 0), _p(keys), _p(ip),
                                    _p(cs), _p(xf),
                                    ctypes.c_int64(max(cap, 1)), ctypes.c_int64(grid + 1), _p(n_out), _p(g_out))
        _check(st, "cube_pp_bin_tile")
        N = int(n_out[0])
        return dict(keys=keys[:N].copy(), ip=ip[:N].copy(), cell_start=cs[: int(g_out[0]) + 1].copy(),
                    xf=xf[: 3 * N].reshape(3, N).copy(), N=N)

    def pp_pair_count(self, img: Image, ires, ixyz3, apm3, ratio_sf) -> int:
        """Ordered PP pairs with 0 < r < range evaluated by the kick (algorithmic work)."""
        out = np.zeros(1, np.int64)
        ires, ixyz3, ratio_sf, apm3 = _c32(ires), _c32(ixyz3), _c32(ratio_sf), _f32(apm3)
        st = lib().cube_pp_pair_count(_p(ires), _p(ixyz3), _p(apm3), _p(ratio_sf), _p(img.rhoc), _p(img.idx_b_r),
                                      _p(img.xp), _p(out))
        _check(st, "cube_pp_pair_count")
        return int(out[0])

    def stage_times(self):
        ms = np.zeros(4, np.float32)
        _check(lib().cube_stage_times(_p(ms)), "cube_stage_times")
        return ms

    @staticmethod
    def enable_timing(on: bool):
        lib().cube_enable_timing(ctypes.c_int(1 if on else 0))

    @staticmethod
    def timing_read(max_calls: int = 256) -> np.ndarray:
        """[n][4] stage times (ms) of the timed calls since the last read: PM3, PP binning+list,
        PP force kernel, whole pipeline."""
        ms = np.zeros((max_calls, 4), np.float32)
        n = np.zeros(1, np.int32)
        _check(lib().cube_timing_read(_p(ms), ctypes.c_int32(max_calls), _p(n)), "cube_timing_read")
        return ms[: int(n[0])].copy()

    @staticmethod
    def launch_count() -> int:
        f = lib().cube_launch_count
        f.restype = ctypes.c_int64
        return int(f())

    @staticmethod
    def fp32_peak_tflops() -> float:
        t = np.zeros(1, np.float32)
        _check(lib().cube_fp32_peak_probe(_p(t)), "cube_fp32_peak_probe")
        return float(t[0])

    @staticmethod
    def finalize():
        lib().c_gpu_velocity_finalize()
        lib().c_pm3_fft_finalize()


def green_table(n: int, apm_soft: float, apm_range: float, gridsize: float) -> np.ndarray:
    """Green_3D (Green.f90:1-80) tabulated in FP64 on the device -> float32 [n][n][n/2+1]."""
    G = np.zeros((n, n, n // 2 + 1), np.float32)
    _check(lib().cube_green_table(ctypes.c_int32(n), ctypes.c_float(apm_soft), ctypes.c_float(apm_range),
                                  ctypes.c_float(gridsize), _p(G)), "cube_green_table")
    return G


def force_truth_fp64(pos: np.ndarray, box: float, app: float, targets: np.ndarray, tol: float = 1e-9):
    """FP64 Ewald-split periodic softened force on `targets` (device); returns float64 [nt,3]."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    targets = np.ascontiguousarray(targets, dtype=np.int64)
    rcut = 0.5 * box
    alpha = np.sqrt(-np.log(tol)) / rcut
    kmax = 2.0 * alpha * np.sqrt(-np.log(tol))
    nmax = int(np.ceil(kmax * box / (2 * np.pi)))
    F = np.zeros((targets.shape[0], 3), np.float64)
    _check(lib().cube_force_truth_fp64(_p(pos), ctypes.c_int64(pos.shape[0]), ctypes.c_double(box),
                                       ctypes.c_double(app), _p(targets), ctypes.c_int64(targets.shape[0]),
                                       ctypes.c_double(alpha), ctypes.c_double(rcut), ctypes.c_int32(nmax), _p(F)),
           "cube_force_truth_fp64")
    return F
