"""cube_pp_force_noalloc: the PP kick for callers that cannot let the library allocate device
memory (their own pool owns all of it, or an allocation-free policy is in force).  It must give
the same kick as the regular entry point, call after call, while using only the caller's buffers
and the library's static scratch array."""
import ctypes

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

SIXPI = np.float32(6 * np.pi)
TOL = 1e-5  # relative rms of the velocity change, as in the PP parity tests


def _tables(L):
    from cube2_b200.layout import RATIO_SF, apm3_table, ixyz3_table
    return (np.arange(1, L.ns3 + 1, dtype=np.int32), np.full(L.ns3, 2, np.int32), ixyz3_table(L), apm3_table(4.0),
            RATIO_SF.copy())


def _noalloc(img, isort, ires, ix, apm3, rs, d_rhoc, d_idx, d_xp, d_vp, d_out, n_used=None, stream=None):
    from cube2_b200.kick import _p, lib
    f = lib().cube_pp_force_noalloc
    return f(_p(isort), _p(ires), _p(ix), _p(apm3), _p(rs), ctypes.c_void_p(d_rhoc.data_ptr()),
             ctypes.c_void_p(d_idx.data_ptr()), ctypes.c_void_p(d_xp.data_ptr()),
             ctypes.c_int64(img.n_used if n_used is None else n_used), ctypes.c_void_p(d_vp.data_ptr()),
             ctypes.c_float(1.0), ctypes.c_float(SIXPI), ctypes.c_float(1.0), ctypes.c_void_p(d_out.data_ptr()),
             None if stream is None else ctypes.c_void_p(stream.cuda_stream))


def _case(name):
    if name == "zeldovich64":
        from cube2_b200 import workloads as W
        return W.make("zeldovich64")
    return load_golden(name)[0]


@pytest.mark.parametrize("name", ["t32_edge", "zeldovich64"])
def test_noalloc_matches_regular_entry_point_twice(gpu, name):
    import torch
    from cube2_b200.kick import FineKick
    img = _case(name)
    L = img.layout
    fk = FineKick(L)
    isort, ires, ix, apm3, rs = _tables(L)
    want, f2, vmax, _, _ = fk.c_pp_force_kernel(img, isort, ires, ix, apm3, rs, 1.0, SIXPI, 1.0)
    dwant = (want - img.vp).astype(np.float64)
    dev = torch.device("cuda:0")
    d_rhoc = torch.from_numpy(img.rhoc.reshape(-1).copy()).to(dev)
    d_idx = torch.from_numpy(img.idx_b_r.reshape(-1).copy()).to(dev)
    d_xp = torch.from_numpy(img.xp.reshape(-1).copy()).to(dev)
    vp0 = torch.from_numpy(img.vp.reshape(-1).copy()).to(dev)
    torch.cuda.synchronize()
    side = torch.cuda.Stream(device=dev)
    for call in range(3):  # the shared scratch keeps the previous call's contents
        d_vp = vp0.clone()
        d_out = torch.full((8,), 7.0, dtype=torch.float32, device=dev)
        torch.cuda.synchronize()
        # the third call runs on a stream of the caller's
        st = _noalloc(img, isort, ires, ix, apm3, rs, d_rhoc, d_idx, d_xp, d_vp, d_out,
                      stream=side if call == 2 else None)
        assert st == 0
        torch.cuda.synchronize()
        got = d_vp.cpu().numpy().reshape(-1, 3)
        dgot = (got - img.vp).astype(np.float64)
        assert np.sqrt(np.sum((dgot - dwant) ** 2) / np.sum(dwant ** 2)) < TOL, call
        assert np.all(got[~img.active] == img.vp[~img.active])
        o = d_out.cpu().numpy()
        assert o[5:6].view(np.int32)[0] == 0
        assert abs(o[1] - f2) <= TOL * f2
        np.testing.assert_allclose(o[2:5], vmax, rtol=TOL)


def test_noalloc_rejects_inputs_beyond_its_scratch(gpu):
    import torch
    from cube2_b200.kick import FineKick, lib
    img, _ = load_golden("t32")
    L = img.layout
    FineKick(L)
    isort, ires, ix, apm3, rs = _tables(L)
    dev = torch.device("cuda:0")
    t = torch.zeros(16, dtype=torch.float32, device=dev)
    too_many = 524288 + 1  # CUBE_NOALLOC_MAX_PARTICLES + 1
    st = _noalloc(img, isort, ires, ix, apm3, rs, t, t, t, t, t, n_used=too_many)
    assert st == 5  # CUBE_ERR_CAPACITY, nothing launched
    assert lib().cube_last_error() == 5


@pytest.mark.parametrize("geom", [(128, 1, 2), (80, 5, 2), (256, 2, 2)])
def test_noalloc_rejects_layouts_beyond_its_scratch(gpu, geom):
    """More PP cells than CUBE_NOALLOC_MAX_CELLS (a 128^3 tile: 68^3 PP cells), more than 64
    tiles (5^3), more coarse cells over the extended tiles than CUBE_NOALLOC_MAX_CELLS
    (8 x 34^3): rejected with CUBE_ERR_CAPACITY before anything is launched."""
    import torch
    from cube2_b200.kick import FineKick, lib
    from cube2_b200.layout import Layout
    ng, nnt, nns = geom
    L = Layout(ng=ng, nnt=nnt, nns=nns, ratio_cs=4, ngb=4, app=0.1)
    FineKick(L)
    isort, ires, ix, apm3, rs = _tables(L)
    dev = torch.device("cuda:0")
    t = torch.zeros(16, dtype=torch.float32, device=dev)

    class _Img:
        n_used = 1

    st = _noalloc(_Img, isort, ires, ix, apm3, rs, t, t, t, t, t)
    assert st == 5
    assert lib().cube_last_error() == 5
