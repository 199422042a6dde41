"""Drift and buffer rebuild on the GPU (cube_drift_device, cube_drift, cube_buffer_v_device)
against the CPU restatement (oracle/drift_oracle.py, itself pinned to the loop restatement
of drift.f90 and the buffer routines in tests/test_drift.py).  Integer and byte outputs
must match bit for bit: counts, spine, offsets, velocities and particle ids."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIXPI = float(np.float32(6 * np.pi))


def _random_image(ngb, n, seed, vscale, ng=32, nnt=2, sigma=None):
    from cube2_b200 import ic
    from cube2_b200.layout import Layout, build_image
    L = Layout(ng=ng, nnt=nnt, nns=2, ratio_cs=4, ngb=ngb, app=0.1)
    rng = np.random.default_rng(seed)
    if sigma is None:
        pos = rng.random((n, 3)) * ng
    else:
        pos = ic.lognormal_poisson(ng, sigma, seed)[0]
    vel = np.clip(rng.standard_normal((pos.shape[0], 3)) * vscale, -2.7 * L.ncb, 2.7 * L.ncb).astype(np.float32)
    return L, build_image(pos, vel, L)


def _cases():
    from cube2_b200 import workloads as W
    yield "uniform32_ncb1", *_random_image(4, 3000, 11, 1.5), 1.3, False
    yield "uniform32_ncb2", *_random_image(8, 3000, 12, 2.5), 1.3, False
    yield "clustered64", *_random_image(4, 0, 13, 1.0, ng=64, sigma=1.5), 1.0, False
    img = W.make("batch8")
    img.vp[:] = np.clip(img.vp * 40.0, -2.5, 2.5)
    yield "batch8_tile_periodic", img.layout, img, 1.0, True


def _compare(got, want):
    names = ["rhoc", "idx_b_r", "xp", "vp", "pid"]
    for g, w, nm in zip(got, want, names):
        np.testing.assert_array_equal(np.asarray(g).reshape(-1), np.asarray(w).reshape(-1), err_msg=nm)


@pytest.mark.parametrize("case", ["uniform32_ncb1", "uniform32_ncb2", "clustered64", "batch8_tile_periodic"])
def test_device_drift_matches_oracle(gpu, case):
    import torch
    from cube2_b200.drift import DeviceImage
    from cube2_b200.kick import CUBE_PM3_PERIODIC, CUBE_PM3_TILE_PERIODIC, FineKick
    from oracle import drift_oracle as D
    name, L, img, dt_mid, tp = next(c for c in _cases() if c[0] == case)
    vz = float(np.abs(img.vp[:, 2]).max())
    FineKick(L, pm3_mode=CUBE_PM3_TILE_PERIODIC if tp else CUBE_PM3_PERIODIC).configure()
    want = D.drift_image(L, img.rhoc, img.xp, img.vp, img.pid, dt_mid, vz, tile_periodic=tp)
    di = DeviceImage(img, torch.device("cuda:0"))
    di.drift(dt_mid, vz)
    got = di.to_host()
    assert got.n_used == want[2].shape[0] and got.n_particles == want[5]
    _compare((got.rhoc, got.idx_b_r, got.xp, got.vp, got.pid), want[:5])
    # the physical copies hold every particle once
    if not tp:
        phys_pid = np.sort(got.pid[got.active])
        np.testing.assert_array_equal(phys_pid, np.arange(img.n_particles))


def test_host_drift_equals_device_drift(gpu):
    from cube2_b200.drift import drift_host
    from oracle import drift_oracle as D
    name, L, img, dt_mid, tp = next(_cases())
    vz = float(np.abs(img.vp[:, 2]).max())
    out = drift_host(img, dt_mid, vz)
    want = D.drift_image(L, img.rhoc, img.xp, img.vp, img.pid, dt_mid, vz)
    _compare((out.rhoc, out.idx_b_r, out.xp, out.vp, out.pid), want[:5])


def test_capacity_is_reported_and_retry_fits(gpu):
    import torch
    from cube2_b200.drift import _dp
    from cube2_b200.kick import CUBE_PM3_PERIODIC, FineKick, lib
    name, L, img, dt_mid, tp = next(_cases())
    FineKick(L, pm3_mode=CUBE_PM3_PERIODIC).configure()
    dev = torch.device("cuda:0")

    def up(a):
        return torch.from_numpy(np.ascontiguousarray(a).reshape(-1).copy()).to(dev)
    rho, idx, xp, vp = up(img.rhoc), up(img.idx_b_r), up(img.xp), up(img.vp)
    rho2, idx2 = torch.zeros_like(rho), torch.zeros_like(idx)
    small = 10
    xp2 = torch.zeros(3 * small, dtype=torch.int16, device=dev)
    vp2 = torch.zeros(3 * small, dtype=torch.float32, device=dev)
    n_new, n_phys = ctypes.c_int64(), ctypes.c_int64()
    st = lib().cube_drift_device(_dp(rho), _dp(idx), _dp(xp), _dp(vp), None, ctypes.c_int64(img.n_used),
                                 ctypes.c_float(dt_mid), ctypes.c_float(2.0), _dp(rho2), _dp(idx2), _dp(xp2),
                                 _dp(vp2), None, ctypes.c_int64(small), ctypes.byref(n_new), ctypes.byref(n_phys),
                                 None)
    assert st == 5 and n_new.value > small and n_phys.value == img.n_particles
    assert np.all(vp2.cpu().numpy() == 0)  # nothing written past the sizes


def test_buffer_v_matches_oracle(gpu):
    import torch
    from cube2_b200.drift import DeviceImage
    from cube2_b200.kick import CUBE_PM3_PERIODIC, FineKick
    from oracle import drift_oracle as D
    name, L, img, dt_mid, tp = next(_cases())
    FineKick(L, pm3_mode=CUBE_PM3_PERIODIC).configure()
    vp = img.vp.copy()
    vp[img.active] += np.float32(0.25)  # a kick changes the physical copies only
    img.vp = vp
    di = DeviceImage(img, torch.device("cuda:0"))
    di.buffer_v()
    got = di.to_host().vp
    np.testing.assert_array_equal(got, D.buffer_v(L, img.rhoc, vp))


def test_kick_drift_loop_matches_oracle_each_step(gpu):
    """Three steps of kick, buffer_v, drift on a clustered image: every drift equals the
    oracle's drift of the same state, and the particle set is conserved."""
    import torch
    from cube2_b200 import workloads as W
    from cube2_b200.drift import DeviceImage
    from cube2_b200.kick import CUBE_PM3_PERIODIC, FineKick
    from oracle import drift_oracle as D
    img = W.make("zeldovich64")
    L = img.layout
    tabs = W.tables("zeldovich64")
    fk = FineKick(L, pm3_mode=CUBE_PM3_PERIODIC, apm3f=4.0)
    di = DeviceImage(img, torch.device("cuda:0"))
    out = torch.zeros(8, device=di.device)
    for step in range(3):
        fk.kick_fine_device(di.rhoc, di.idx, di.xp, di.n_used, di.vp, out, *tabs, 1.0, SIXPI, 0.01)
        di.buffer_v()
        torch.cuda.synchronize()
        vmax = out[2:5].cpu().numpy()
        vz = float(vmax[2])
        dt_mid = float(min(2.0, 1.6 / float(vmax.max())))  # at most 0.4 coarse cells per step
        before = di.to_host()
        want = D.drift_image(L, before.rhoc, before.xp, before.vp, before.pid, dt_mid, vz)
        di.drift(dt_mid, vz)
        got = di.to_host()
        _compare((got.rhoc, got.idx_b_r, got.xp, got.vp, got.pid), want[:5])
        np.testing.assert_array_equal(np.sort(got.pid[got.active]), np.arange(img.n_particles))


@pytest.mark.parametrize("nw", [32, 64])
def test_power_spectrum_matches_oracle(gpu, nw):
    import torch
    from cube2_b200 import workloads as W
    from cube2_b200.drift import DeviceImage
    from cube2_b200.kick import CUBE_PM3_PERIODIC, FineKick
    from oracle import power_oracle as P
    img = W.make("zeldovich64")
    L = img.layout
    FineKick(L, pm3_mode=CUBE_PM3_PERIODIC).configure()
    di = DeviceImage(img, torch.device("cuda:0"))
    got = di.power_spectrum(nw)
    pos = W.physical_positions(img) / L.ratio_cs  # coarse-cell units
    want = P.power_spectrum(pos, L.nc, nw)
    np.testing.assert_array_equal(got["modes"], want["modes"])
    ok = want["modes"] > 0
    np.testing.assert_allclose(got["k"][ok], want["k"][ok], rtol=1e-12)
    np.testing.assert_allclose(got["pk"][ok], want["pk"][ok], rtol=2e-3, atol=1e-12)
    np.testing.assert_allclose(got["delta2"][ok], want["delta2"][ok], rtol=2e-3, atol=1e-9)


@pytest.mark.parametrize("name", ["uniform32_ncb1", "uniform32_ncb2"])
def test_snapshot_round_trip_rebuilds_the_image(gpu, tmp_path, name):
    """A checkpoint holds the physical particles only; reading it back and rebuilding the
    buffers with a zero-length drift gives the written image bit for bit."""
    from cube2_b200 import snapshot as S
    _, L, img, _, _ = next(c for c in _cases() if c[0] == name)
    prefix, suffix = str(tmp_path) + "/0.000_", "_1.bin"
    S.write(img, prefix, suffix)
    back, h = S.read(L, prefix, suffix)
    assert h["nplocal"] == img.n_particles
    _compare((back.rhoc, back.idx_b_r, back.xp, back.vp, back.pid), (img.rhoc, img.idx_b_r, img.xp, img.vp, img.pid))
