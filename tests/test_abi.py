"""The C-ABI library: symbols, layout configuration and host-side error paths (no GPU needed)."""
import ctypes
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, load_golden


def _declared_functions():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"^\s*(?:void|int64_t|int|const char\s*\*)\s*\*?\s*(\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(cube_lib):
    names = _declared_functions()
    assert "c_pm3_force_kernel" in names and "c_pp_force_kernel" in names
    for n in names:
        assert hasattr(cube_lib, n), n


def test_error_strings(cube_lib):
    cube_lib.cube_error_string.restype = ctypes.c_char_p
    for s in range(8):
        assert len(cube_lib.cube_error_string(s)) > 0


def test_not_configured_is_reported(cube_lib):
    """A fresh process that skips cube_set_layout gets status 2, not an abort."""
    code = ("import ctypes,sys; sys.path.insert(0, %r); from cube2_b200 import kick; L = kick.lib(); "
            "import numpy as np; z = np.zeros(64, np.int32); "
            "s = L.cube_pp_force(*([None]*13), None, None, None); print(s)") % ROOT
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "2"


def test_layout_validation(cube_lib):
    from cube2_b200.kick import CLayout
    bad = [CLayout(30, 2, 2, 4, 4, 0.1, 1, 4.0, 0.0, 2),   # ng not divisible by ratio_cs*nnt
           CLayout(32, 2, 3, 4, 4, 0.1, 1, 4.0, 0.0, 2),   # nt not divisible by nns
           CLayout(32, 2, 2, 4, 2, 0.1, 1, 4.0, 0.0, 2),   # ngb not a multiple of ratio_cs
           CLayout(32, 2, 2, 4, 4, 0.1, 7, 4.0, 0.0, 2),   # unknown PM3 mode
           CLayout(32, 2, 2, 4, 4, 0.1, 1, 4.0, 0.0, 1)]   # CIC assignment not provided
    for cl in bad:
        assert cube_lib.cube_set_layout(ctypes.byref(cl)) == 1
    good = CLayout(32, 2, 2, 4, 4, 0.1, 1, 4.0, 0.0, 2)
    assert cube_lib.cube_set_layout(ctypes.byref(good)) == 0
    got = CLayout()
    assert cube_lib.cube_get_layout(ctypes.byref(got)) == 0
    assert (got.ng, got.nnt, got.nns, got.ngb, got.pm3_mode) == (32, 2, 2, 4, 1)


def test_pp_shape_table_and_index_check(cube_lib):
    """The PP kernel shape table is readable without a GPU; a shape index outside it is refused."""
    from cube2_b200 import kick as K
    table, cur = K.pp_shapes()
    assert len(table) >= 8 and table[0]["chunk"] == 16 and 0 <= cur < len(table)
    assert all(t["chunk"] in (4, 8, 16, 32) and t["jtile"] % 32 == 0 and t["unroll"] >= 1 for t in table)
    # both pair-law forms: packed f32x2 (the default, shape 0) and scalar FP32
    assert table[0]["packed"] == 1 and {t["packed"] for t in table} == {0, 1}
    for bad in (-2, len(table)):
        with pytest.raises(K.CubeError):
            K.pp_set_shape(bad)
    K.pp_set_shape(len(table) - 1)
    K.pp_set_shape(-1)


def _call_pp(fk, img, ires, ixyz3, idx_b_r=None, rhoc=None):
    from cube2_b200.kick import _p
    from cube2_b200.layout import RATIO_SF, apm3_table
    L = img.layout
    vp = img.vp.copy()
    f2 = np.zeros(1, np.float32)
    vmax = np.zeros(3, np.float32)
    pt = np.zeros(L.ns3)
    tt = np.zeros(L.ns3)
    isort = np.arange(1, L.ns3 + 1, dtype=np.int32)
    apm3 = apm3_table(4.0)
    rs = RATIO_SF.copy()
    idx_b_r = img.idx_b_r if idx_b_r is None else idx_b_r
    rhoc = img.rhoc if rhoc is None else rhoc
    from cube2_b200.kick import lib
    return lib().cube_pp_force(_p(isort), _p(np.ascontiguousarray(ires, np.int32)),
                               _p(np.ascontiguousarray(ixyz3, np.int32)), _p(apm3), _p(rs), _p(rhoc), _p(idx_b_r),
                               _p(img.xp), _p(vp), ctypes.c_float(1.0), ctypes.c_float(1.0), ctypes.c_float(1.0),
                               _p(f2), _p(vmax), _p(pt), _p(tt))


def test_invalid_metadata_returns_status_without_device(cube_lib):
    """Bad ires / ixyz3 / spine are rejected on the host (the reference calls exit():
    pp_force_kernel.cu:985-986, pm3_fft_cuda.cu:537-539)."""
    from cube2_b200.kick import FineKick
    from cube2_b200.layout import ixyz3_table
    img, _ = load_golden("t32")
    L = img.layout
    FineKick(L)
    ix = ixyz3_table(L)
    ires = np.full(L.ns3, 2, np.int32)
    bad_ires = ires.copy()
    bad_ires[5] = 7
    assert _call_pp(None, img, bad_ires, ix) == 1
    bad_ix = ix.copy()
    bad_ix[3, 0] = L.nns + 1
    assert _call_pp(None, img, ires, bad_ix) == 1
    dup = ix.copy()
    dup[1] = dup[0]
    assert _call_pp(None, img, ires, dup) == 1
    bad_idx = img.idx_b_r.copy()
    bad_idx.reshape(-1)[10] += 1
    assert _call_pp(None, img, ires, ix, idx_b_r=bad_idx) == 1
    neg = img.rhoc.copy()
    neg.reshape(-1)[7] = -1
    assert _call_pp(None, img, ires, ix, rhoc=neg) == 1


def test_valid_call_without_gpu_reports_no_device(cube_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from cube2_b200.kick import FineKick
    from cube2_b200.layout import ixyz3_table
    img, _ = load_golden("t32")
    FineKick(img.layout)
    st = _call_pp(None, img, np.full(img.layout.ns3, 2, np.int32), ixyz3_table(img.layout))
    assert st in (3, 6)


def test_device_kick_pointer_checks_without_device(cube_lib):
    """cube_kick_fine_device: an image without particles may pass null particle arrays (the call
    then goes on to the device), while n_used > 0 with a null particle array is refused on the
    host as an invalid argument."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from cube2_b200.kick import FineKick, _p
    from cube2_b200.layout import RATIO_SF, apm3_table, ixyz3_table
    img, _ = load_golden("t32")
    L = img.layout
    FineKick(L)
    isort = np.arange(1, L.ns3 + 1, dtype=np.int32)
    ires = np.full(L.ns3, 2, np.int32)
    ix = np.ascontiguousarray(ixyz3_table(L), np.int32)
    apm3, rs = apm3_table(4.0), RATIO_SF.copy()
    out = np.zeros(8, np.float32)  # stands in for device memory: the checks only test for NULL
    gk = (ctypes.c_void_p * 5)()

    def call(xp, n_used, vp):
        return cube_lib.cube_kick_fine_device(_p(isort), _p(ires), _p(ix), _p(apm3), _p(rs), _p(img.rhoc),
                                              _p(img.idx_b_r), xp, ctypes.c_int64(n_used), gk, vp,
                                              ctypes.c_float(1.0), ctypes.c_float(1.0), ctypes.c_float(1.0),
                                              _p(out), None)

    assert call(None, 0, None) in (3, 6)  # past the checks, no device
    assert call(None, 5, _p(out)) == 1
    assert call(_p(img.xp), 5, None) == 1
    assert call(_p(img.xp), -1, _p(out)) == 1


def test_graph_create_pointer_checks_without_device(cube_lib):
    """cube_kick_graph_create applies the same pointer checks as the device kick it captures."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from cube2_b200.kick import CUBE_PM3_PERIODIC, FineKick, _p
    from cube2_b200.layout import RATIO_SF, apm3_table, ixyz3_table
    img, _ = load_golden("t32")
    L = img.layout
    FineKick(L, pm3_mode=CUBE_PM3_PERIODIC)
    isort = np.arange(1, L.ns3 + 1, dtype=np.int32)
    ires = np.full(L.ns3, 2, np.int32)
    ix = np.ascontiguousarray(ixyz3_table(L), np.int32)
    apm3, rs = apm3_table(4.0), RATIO_SF.copy()
    out = np.zeros(8, np.float32)  # stands in for device memory: the checks only test for NULL

    def call(xp, n_used, vp):
        h = ctypes.c_void_p()
        st = cube_lib.cube_kick_graph_create(_p(isort), _p(ires), _p(ix), _p(apm3), _p(rs), _p(img.rhoc),
                                             _p(img.idx_b_r), xp, ctypes.c_int64(n_used), vp,
                                             ctypes.c_float(1.0), ctypes.c_float(1.0), ctypes.c_float(1.0),
                                             _p(out), ctypes.byref(h))
        assert not h.value  # no graph on failure
        return st

    assert call(None, 0, None) in (3, 6)  # past the checks, no device
    assert call(None, 5, _p(out)) == 1
    assert call(_p(img.xp), 5, None) == 1
