"""FP64 conservation sums of a kick (cube_kick_sums), reduced on the device.

* The device sums equal the FP64 sums of the same velocity arrays taken on the host.
* PP conserves momentum: every pair is evaluated from both sides with dx and -dx, so the
  PP forces of the physical particles of a periodic image cancel up to FP32 rounding.
* PM3 on a periodic mesh conserves momentum too: TSC deposit and gather are the same
  operator and the 4-point difference is antisymmetric, so sum_i F_i = rho^T A rho with A
  antisymmetric.  Its sums also match the CPU restatement's.
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

SIXPI = float(np.float32(6 * np.pi))


def _device(img):
    import torch
    dev = torch.device("cuda:0")
    return (torch.from_numpy(img.rhoc.reshape(-1).copy()).to(dev), torch.from_numpy(img.idx_b_r.reshape(-1).copy()).to(dev),
            dev)


def _host_sums(img, va, vb, mass=1.0):
    act = img.active
    a = va[act].astype(np.float64)
    b = vb[act].astype(np.float64)
    dm = mass * (b - a)
    return dm.sum(axis=0), float(0.5 * mass * np.sum(b * b - a * a)), np.abs(dm).sum(axis=0), int(act.sum())


def _image(name):
    if name == "zeldovich64":
        from cube2_b200 import workloads as W
        return W.make("zeldovich64")
    if name == "clumpy64":
        from cube2_b200 import ic
        from cube2_b200.layout import Layout, build_image
        from oracle.layouts import LAYOUTS
        return build_image(*ic.lognormal_poisson(64, 1.5, 4100)[:2], Layout(**LAYOUTS["cfg0"]))
    return load_golden(name)[0]


@pytest.mark.parametrize("name", ["t32", "zeldovich64"])
def test_device_sums_equal_host_fp64_sums(gpu, name):
    import torch
    from cube2_b200.kick import FineKick, kick_sums
    from cube2_b200.layout import RATIO_SF, apm3_table, ixyz3_table
    img = _image(name)
    L = img.layout
    fk = FineKick(L)
    vb, _ = fk.kick_fine(img, np.arange(1, L.ns3 + 1, dtype=np.int32), np.full(L.ns3, 2, np.int32), ixyz3_table(L),
                         apm3_table(4.0), RATIO_SF, 1.0, SIXPI, 1.0)
    d_rhoc, d_idx, dev = _device(img)
    va_d = torch.from_numpy(img.vp.reshape(-1).copy()).to(dev)
    vb_d = torch.from_numpy(vb.reshape(-1).copy()).to(dev)
    s = kick_sums(d_rhoc, d_idx, img.n_used, va_d, vb_d, mass=2.0)
    p, ke, scale, n = _host_sums(img, img.vp, vb, mass=2.0)
    assert s["particles"] == n == img.n_particles
    np.testing.assert_allclose(s["momentum"], p, rtol=1e-9, atol=1e-12 * scale.max())
    np.testing.assert_allclose(s["momentum_scale"], scale, rtol=1e-12)
    assert abs(s["kinetic_energy"] - ke) <= 1e-9 * abs(ke)


@pytest.mark.parametrize("name", ["zeldovich64", "clumpy64"])
def test_pp_and_pm3_conserve_momentum(gpu, name):
    import torch
    from cube2_b200.kick import CUBE_PM3_PERIODIC, FineKick, kick_sums
    from cube2_b200.layout import RATIO_SF, apm3_table, ixyz3_table
    from oracle import oracle as O
    img = _image(name)
    L = img.layout
    tabs = (np.arange(1, L.ns3 + 1, dtype=np.int32), np.full(L.ns3, 2, np.int32), ixyz3_table(L))
    fk = FineKick(L, pm3_mode=CUBE_PM3_PERIODIC, apm3f=4.0)
    zero = np.zeros_like(img.vp)
    v_pm3, _, _, _ = fk.c_pm3_force_kernel(img, *tabs, RATIO_SF, 1.0, SIXPI, 1.0, vp=zero.copy())
    v_pp, _, _, _, _ = fk.c_pp_force_kernel(img, *tabs, apm3_table(4.0), RATIO_SF, 1.0, SIXPI, 1.0,
                                            vp=zero.copy())
    d_rhoc, d_idx, dev = _device(img)
    z = torch.zeros(zero.size, dtype=torch.float32, device=dev)
    s_pm3 = kick_sums(d_rhoc, d_idx, img.n_used, z, torch.from_numpy(v_pm3.reshape(-1).copy()).to(dev))
    s_pp = kick_sums(d_rhoc, d_idx, img.n_used, z, torch.from_numpy(v_pp.reshape(-1).copy()).to(dev))
    for s in (s_pm3, s_pp):
        assert np.all(s["momentum_scale"] > 0)
        assert np.all(np.abs(s["momentum"]) <= 1e-5 * s["momentum_scale"]), (s["momentum"], s["momentum_scale"])
    # PM3's sums against the restatement's (FP64 deposit, FFT and gather)
    G = O.green(L.ng * 2, 4.0, 0.0, 0.5)
    ref = O.pm3_periodic(img, 2, G, 1.0, SIXPI, 1.0)
    p, ke, scale, _ = _host_sums(img, zero, ref["dv"])
    assert np.all(np.abs(s_pm3["momentum"] - p) <= 1e-5 * scale)
    assert abs(s_pm3["kinetic_energy"] - ke) <= 1e-5 * abs(ke)
