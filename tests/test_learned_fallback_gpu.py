"""Per-cell check and fallback of the learned PP shell (cube_learned_fallback).

The full-cutoff kick (PM3 + PP at cutoff 2, the plain method) is the reference for the
network: every coarse cell with physical particles is checked on its first few particles, and
a cell whose learned velocity change differs from the full-cutoff one by more than the bound
(relative rms) is recomputed at cutoff 2, i.e. takes the full-cutoff velocities.  After the
fallback every checked cell is within the bound.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIXPI = float(np.float32(6 * np.pi))
BOUND = 0.01


def _interior_cells(img):
    """(first storage index, count) of every interior coarse cell, in the kernel's order."""
    L = img.layout
    r = img.rhoc.reshape(L.nnt ** 3, L.nte, L.nte, L.nte).astype(np.int64)
    idx = img.idx_b_r.reshape(L.nnt ** 3, L.nte, L.nte)
    tail = np.cumsum(r[..., ::-1], axis=-1)[..., ::-1]  # sum over i' >= i
    base = idx[..., None] - tail
    s = slice(L.ncb, L.ncb + L.nt)
    return base[:, s, s, s].reshape(-1), r[:, s, s, s].reshape(-1)


@pytest.fixture(scope="module")
def kicked():
    import torch
    from cube2_b200 import ic
    from cube2_b200 import learned as Ln
    from cube2_b200.kick import CUBE_PM3_PERIODIC, FineKick
    from cube2_b200.layout import Layout, build_image, ixyz3_table
    from oracle.layouts import LAYOUTS
    img = build_image(*ic.lognormal_poisson(64, 1.5, 4100)[:2], Layout(**LAYOUTS["cfg0"]))
    L = img.layout
    dev = torch.device("cuda:0")
    rho, idx, xp, vp0 = Ln.device_image(img, dev)
    tabs = (np.arange(1, L.ns3 + 1, dtype=np.int32), np.full(L.ns3, 2, np.int32), ixyz3_table(L))
    out = torch.zeros(8, device=dev)
    vpf = vp0.clone()
    from cube2_b200.layout import RATIO_SF, apm3_table
    FineKick(L, pm3_mode=CUBE_PM3_PERIODIC, apm3f=Ln.PLAIN.apm3f).kick_fine_device(
        rho, idx, xp, img.n_used, vpf, out, *tabs, apm3_table(Ln.PLAIN.apm3f), RATIO_SF, 1.0, SIXPI, 1.0)
    torch.cuda.synchronize()
    return img, (rho, idx, xp, vp0, vpf), tabs


def test_cells_over_the_bound_fall_back_to_the_full_cutoff_kick(gpu, kicked):
    """A learned result with a 5 % error in chosen cells and 0.1 % elsewhere: exactly the chosen
    cells fall back, their particles get the full-cutoff velocities bit for bit, the others keep
    the learned ones, and a second check finds every cell within the bound."""
    import torch
    from cube2_b200 import learned as Ln
    img, (rho, idx, xp, vp0, vpf), _ = kicked
    base, cnt = _interior_cells(img)
    rng = np.random.default_rng(7)
    bad = (rng.random(cnt.size) < 0.3) & (cnt > 0)
    dv = (vpf - vp0).cpu().numpy().reshape(-1, 3)
    noise = rng.standard_normal(dv.shape).astype(np.float32)
    scale = np.full(dv.shape[0], 1e-3, np.float32)
    for b, c in zip(base[bad], cnt[bad]):
        scale[b:b + c] = 5e-2
    mag = np.linalg.norm(dv, axis=1, keepdims=True)
    vpl = (vp0.cpu().numpy().reshape(-1, 3) + dv + noise * scale[:, None] * mag / np.sqrt(3)).astype(np.float32)
    d_vpl = torch.from_numpy(vpl.reshape(-1)).to(vp0.device)
    d_out = torch.zeros_like(d_vpl)
    st = Ln.fallback(rho, idx, img.n_used, vp0, d_vpl, vpf, BOUND, samples=4, d_vp_out=d_out)
    assert st["cells_checked"] == int((cnt > 0).sum())
    assert st["cells_over"] == int(bad.sum())
    assert st["particles_fallen_back"] == int(cnt[bad].sum())
    got = d_out.cpu().numpy().reshape(-1, 3)
    full = vpf.cpu().numpy().reshape(-1, 3)
    for b, c, is_bad in zip(base[cnt > 0], cnt[cnt > 0], bad[cnt > 0]):
        want = full if is_bad else vpl
        np.testing.assert_array_equal(got[b:b + c], want[b:b + c])
    again = Ln.fallback(rho, idx, img.n_used, vp0, d_out, vpf, BOUND, samples=4, d_vp_out=torch.zeros_like(d_out))
    assert again["cells_over"] == 0 and again["sampled_rms_vs_full"] < BOUND


def test_learned_kick_with_fallback_is_within_the_bound(gpu, kicked):
    """The learned kick itself (cutoff-1 split + an untrained network, far off): the cells over
    the bound are recomputed at cutoff 2, after which every checked cell is within the bound
    and the kick's error against the full-cutoff kick is below the bound."""
    import torch
    from cube2_b200 import learned as Ln
    from cube2_b200.kick import CUBE_PM3_PERIODIC, FineKick
    from cube2_b200.layout import RATIO_SF, apm3_table
    img, (rho, idx, xp, vp0, vpf), tabs = kicked
    L = img.layout
    shell = Ln.ShellNet(batch_cap=16, seed=3)
    try:
        vpl = vp0.clone()
        out = torch.zeros(8, device=vp0.device)
        FineKick(L, pm3_mode=CUBE_PM3_PERIODIC, apm3f=Ln.SHORT.apm3f).kick_fine_device(
            rho, idx, xp, img.n_used, vpl, out, *tabs, apm3_table(Ln.SHORT.apm3f), RATIO_SF, 1.0, SIXPI, 1.0)
        shell.kick(rho, idx, xp, img.n_used, vpl, 0.05, SIXPI, 1.0)
        torch.cuda.synchronize()
        before = vpl.clone()
        st = Ln.fallback(rho, idx, img.n_used, vp0, vpl, vpf, BOUND, samples=4)
    finally:
        shell.close()
    assert st["cells_over"] > 0 and st["sampled_rms_vs_full"] > BOUND
    again = Ln.fallback(rho, idx, img.n_used, vp0, vpl, vpf, BOUND, samples=4, d_vp_out=torch.zeros_like(vpl))
    assert again["cells_over"] == 0 and again["sampled_rms_vs_full"] < BOUND
    act = img.active

    def rel(v):
        d_l = (v - vp0).cpu().numpy().reshape(-1, 3)[act].astype(np.float64)
        d_f = (vpf - vp0).cpu().numpy().reshape(-1, 3)[act].astype(np.float64)
        return np.sqrt(np.sum((d_l - d_f) ** 2) / np.sum(d_f ** 2))
    assert rel(vpl) < rel(before)
