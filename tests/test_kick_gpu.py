"""The whole fine-scale kick: fused call == PM3 then PP, device API == host API, and the
force of PM3 + PP against the FP64 direct-summation truth."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

SIXPI = np.float32(6 * np.pi)


def _tables(L):
    from cube2_b200.layout import RATIO_SF, apm3_table, ixyz3_table
    return (np.arange(1, L.ns3 + 1, dtype=np.int32), np.full(L.ns3, 2, np.int32), ixyz3_table(L), apm3_table(4.0),
            RATIO_SF)


def test_kick_fine_equals_pm3_then_pp(gpu):
    from cube2_b200.kick import FineKick
    img, _ = load_golden("t32_edge")
    L = img.layout
    fk = FineKick(L)
    isort, ires, ix, apm3, rs = _tables(L)
    v1, f2a, _, _ = fk.c_pm3_force_kernel(img, isort, ires, ix, rs, 1.0, SIXPI, 1.0)
    v2, f2b, vmax, _, _ = fk.c_pp_force_kernel(img, isort, ires, ix, apm3, rs, 1.0, SIXPI, 1.0, vp=v1.copy())
    v3, out = fk.kick_fine(img, isort, ires, ix, apm3, rs, 1.0, SIXPI, 1.0)
    # the PM3 deposit accumulates with float atomics: runs agree to rounding, not bit for bit
    d2, d3 = (v2 - img.vp).astype(np.float64), (v3 - img.vp).astype(np.float64)
    assert np.sqrt(np.sum((d3 - d2) ** 2) / np.sum(d2 ** 2)) < 1e-6
    assert abs(out[0] - f2a) <= 1e-5 * f2a and abs(out[1] - f2b) <= 1e-6 * f2b
    np.testing.assert_allclose(out[2:], vmax, rtol=1e-5)


def _many_tiles():
    """125 parent tiles: more than the host kick's per-tile events, so it takes the one-piece
    path (whole-array copies, one PP launch)."""
    from cube2_b200 import ic
    from cube2_b200.layout import Layout, build_image
    L = Layout(ng=80, nnt=5, nns=2, ratio_cs=4, ngb=4, app=0.1)
    pos, vel = ic.uniform_random(20000, 80.0, 17)
    return build_image(pos, vel, L)


@pytest.mark.parametrize("case", ["t32", "many_tiles"])
def test_device_api_equals_host_api(gpu, case):
    import torch
    from cube2_b200.kick import FineKick
    img = load_golden("t32")[0] if case == "t32" else _many_tiles()
    L = img.layout
    fk = FineKick(L)
    isort, ires, ix, apm3, rs = _tables(L)
    vh, out_h = fk.kick_fine(img, isort, ires, ix, apm3, rs, 1.0, SIXPI, 1.0)
    dev = torch.device("cuda:0")
    d_rhoc = torch.from_numpy(img.rhoc.reshape(-1).copy()).to(dev)
    d_idx = torch.from_numpy(img.idx_b_r.reshape(-1).copy()).to(dev)
    d_xp = torch.from_numpy(img.xp.reshape(-1).copy()).to(dev)
    d_vp = torch.from_numpy(img.vp.reshape(-1).copy()).to(dev)
    d_out = torch.zeros(8, dtype=torch.float32, device=dev)
    s = torch.cuda.Stream(dev)
    fk.kick_fine_device(d_rhoc, d_idx, d_xp, img.n_used, d_vp, d_out, isort, ires, ix, apm3, rs, 1.0, SIXPI, 1.0,
                        stream=s)
    torch.cuda.synchronize()
    vd = d_vp.cpu().numpy().reshape(-1, 3)
    d_h, d_d = (vh - img.vp).astype(np.float64), (vd - img.vp).astype(np.float64)
    assert np.sqrt(np.sum((d_d - d_h) ** 2) / np.sum(d_h ** 2)) < 1e-6
    o = d_out.cpu().numpy()
    np.testing.assert_allclose(o[:5], out_h, rtol=1e-5)
    assert o[5:6].view(np.int32)[0] == 0


def test_kick_vs_fp64_truth_zeldovich(gpu):
    """64^3 Zel'dovich lattice, PM3 128^3 + PP cutoff 2 cells: rms force error < 1% vs FP64 Ewald,
    and the device FP64 truth agrees with the CPU one."""
    from cube2_b200 import ic
    from cube2_b200.kick import FineKick, force_truth_fp64
    from cube2_b200.layout import Layout, build_image, encode_positions
    from oracle import oracle as O
    from oracle.layouts import LAYOUTS
    L = Layout(**LAYOUTS["cfg0"])
    pos, vel, _ = ic.zeldovich_lattice(64, 0.5, 1000)
    img = build_image(pos, vel, L)
    fk = FineKick(L)
    isort, ires, ix, apm3, rs = _tables(L)
    zero = np.zeros_like(img.vp)
    v, _ = fk.kick_fine(img, isort, ires, ix, apm3, rs, 1.0, SIXPI, 1.0, vp=zero.copy())
    kick = float(np.float32(SIXPI) / np.float32(6.0)) / np.pi
    cc, u = encode_positions(pos, 4, 16)
    posq = (cc + (u.astype(np.float64) + 0.5) / 65536.0) * 4.0
    act = np.nonzero(img.active)[0]
    samp = np.random.default_rng(1).choice(act, 1000, replace=False)
    Fd = force_truth_fp64(posq, 64.0, 0.1, img.pid[samp])
    Fc = O.ewald(posq, 64.0, 0.1, img.pid[samp][:100])
    assert np.max(np.abs(Fd[:100] - Fc)) / np.sqrt(np.mean(Fc ** 2)) < 1e-9
    F = v[samp].astype(np.float64) / kick
    rel = np.sqrt(np.sum((F - Fd) ** 2) / np.sum(Fd ** 2))
    assert rel < 0.01, rel


def test_host_kick_rejects_an_inconsistent_spine_and_recovers(gpu):
    """A spine row that disagrees with its rhoc row makes the host call return
    CUBE_ERR_INVALID without kicking or writing vp, and the next valid call gives the usual
    kick."""
    import dataclasses
    from cube2_b200.kick import CubeError, FineKick
    img, _ = load_golden("t32")
    L = img.layout
    fk = FineKick(L)
    isort, ires, ix, apm3, rs = _tables(L)
    want, out_want = fk.kick_fine(img, isort, ires, ix, apm3, rs, 1.0, SIXPI, 1.0)
    bad_idx = img.idx_b_r.copy()
    rows = L.nte * L.nte
    bad_idx.reshape(-1)[rows // 2] += 1  # an inner row of tile 0: the tile ends stay consistent
    bad = dataclasses.replace(img, idx_b_r=bad_idx)
    vp = img.vp.copy()
    with pytest.raises(CubeError):
        fk.kick_fine(bad, isort, ires, ix, apm3, rs, 1.0, SIXPI, 1.0, vp=vp)
    np.testing.assert_array_equal(vp, img.vp)  # nothing was written back
    got, out_got = fk.kick_fine(img, isort, ires, ix, apm3, rs, 1.0, SIXPI, 1.0)
    d_w, d_g = (want - img.vp).astype(np.float64), (got - img.vp).astype(np.float64)
    assert np.sqrt(np.sum((d_g - d_w) ** 2) / np.sum(d_w ** 2)) < 1e-6


def _device_kick(img, fk, tables):
    import torch
    dev = torch.device("cuda:0")
    d_rhoc = torch.from_numpy(img.rhoc.reshape(-1).copy()).to(dev)
    d_idx = torch.from_numpy(img.idx_b_r.reshape(-1).copy()).to(dev)
    d_xp = torch.from_numpy(img.xp.reshape(-1).copy()).to(dev)
    d_vp = torch.from_numpy(img.vp.reshape(-1).copy()).to(dev)
    d_out = torch.zeros(8, dtype=torch.float32, device=dev)
    fk.kick_fine_device(d_rhoc, d_idx, d_xp, img.n_used, d_vp, d_out, *tables, 1.0, SIXPI, 1.0)
    torch.cuda.synchronize()
    return d_vp.cpu().numpy().reshape(-1, 3), d_out.cpu().numpy()


def test_periodic_kick_with_empty_tiles(gpu):
    """Particles in the middle of two of the eight parent tiles only (more than a coarse cell
    from every tile face, so no buffer copies either): the host kick's tile groups include
    empty ones (nothing to copy, no PP items, bricks without particles), and it must equal the
    device kick; PM3 alone equals the restatement."""
    from cube2_b200 import ic
    from cube2_b200.kick import CUBE_PM3_PERIODIC, FineKick
    from cube2_b200.layout import Layout, build_image
    from oracle import oracle as O
    L = Layout(ng=32, nnt=2, nns=2, ratio_cs=4, ngb=4, app=0.1)
    a, va = ic.uniform_random(3000, 8.0, 21)
    b, vb = ic.uniform_random(3000, 8.0, 22)
    a = a + 4.0                             # tile (0, 0, 0)
    b = b + np.array([20.0, 4.0, 20.0])     # tile (1, 0, 1)
    img = build_image(np.concatenate([a, b]), np.concatenate([va, vb]), L)
    idx = img.idx_b_r.reshape(8, -1)[:, -1]
    assert list(np.diff(np.concatenate([[0], idx]))) == [3000, 0, 0, 0, 0, 3000, 0, 0]
    fk = FineKick(L, pm3_mode=CUBE_PM3_PERIODIC, apm3f=4.0)
    tables = _tables(L)
    isort, ires, ix, apm3, rs = tables
    vh, out_h = fk.kick_fine(img, isort, ires, ix, apm3, rs, 1.0, SIXPI, 1.0)
    vd, out_d = _device_kick(img, fk, tables)
    d_h, d_d = (vh - img.vp).astype(np.float64), (vd - img.vp).astype(np.float64)
    assert np.sum(d_h ** 2) > 0
    assert np.sqrt(np.sum((d_d - d_h) ** 2) / np.sum(d_h ** 2)) < 1e-6
    np.testing.assert_allclose(out_d[:5], out_h, rtol=1e-5)
    assert out_d[5:6].view(np.int32)[0] == 0
    vp, f2, vmax, pt = fk.c_pm3_force_kernel(img, isort, ires, ix, rs, 1.0, SIXPI, 1.0)
    ref = O.pm3_periodic(img, 2, O.green(L.ng * 2, 4.0, 0.0, 0.5), 1.0, SIXPI, 1.0)
    act = img.active
    dv, dr = (vp - img.vp)[act].astype(np.float64), (ref["vp"] - img.vp)[act].astype(np.float64)
    assert np.sqrt(np.sum((dv - dr) ** 2) / np.sum(dr ** 2)) < 1e-5
    assert abs(f2 - ref["f2max"]) <= 1e-5 * ref["f2max"]


def test_periodic_kick_of_an_empty_image(gpu):
    """No particles at all: the host and the device kick return zero maxima and no error."""
    from cube2_b200.kick import CUBE_PM3_PERIODIC, FineKick
    from cube2_b200.layout import Image, Layout
    L = Layout(ng=32, nnt=2, nns=2, ratio_cs=4, ngb=4, app=0.1)
    img = Image(L, np.zeros((0, 3), np.int16), np.zeros((0, 3), np.float32),
                np.zeros((2, 2, 2, L.nte, L.nte, L.nte), np.int32), np.zeros((2, 2, 2, L.nte, L.nte), np.int64),
                np.zeros(0, np.int64), np.zeros(0, bool), 0)
    fk = FineKick(L, pm3_mode=CUBE_PM3_PERIODIC, apm3f=4.0)
    tables = _tables(L)
    vh, out_h = fk.kick_fine(img, *tables, 1.0, SIXPI, 1.0)
    assert vh.size == 0 and np.all(out_h == 0)
    vd, out_d = _device_kick(img, fk, tables)
    assert np.all(out_d[:5] == 0) and out_d[5:6].view(np.int32)[0] == 0
