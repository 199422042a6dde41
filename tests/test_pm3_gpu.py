"""PM3 on the GPU against the CPU restatement of the reference PM3 (kick.f90:403-568).

Both geometries: one periodic image mesh, and the reference's per-subtile
buffered meshes with the caller's Green tables (levels mixed).  Forces agree
within 1e-5 relative rms (FP32 deposit/FFT/gather vs FP64 restatement).
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

SIXPI = np.float32(6 * np.pi)
TOL = 1e-5


def _rel_rms(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


@pytest.mark.parametrize("n,soft,rng_,gs", [(24, 4.0, 7.0, 0.5), (64, 4.0, 0.0, 0.5), (80, 3.5, 7.0, 0.5)])
def test_green_device_fp64_matches_restatement(gpu, n, soft, rng_, gs):
    from cube2_b200.kick import green_table
    from oracle import oracle as O
    G = green_table(n, soft, rng_, gs)
    R = O.green(n, soft, rng_, gs)
    np.testing.assert_allclose(G, R, rtol=2e-6, atol=1e-7 * np.abs(R).max())


@pytest.mark.parametrize("case", ["t32", "t32_edge", "t32b_edge"])
def test_pm3_periodic_matches_restatement(gpu, case):
    from cube2_b200.kick import CUBE_PM3_PERIODIC, FineKick
    from cube2_b200.layout import RATIO_SF, ixyz3_table
    from oracle import oracle as O
    img, _ = load_golden(case)
    L = img.layout
    fk = FineKick(L, pm3_mode=CUBE_PM3_PERIODIC, apm3f=4.0)
    isort = np.arange(1, L.ns3 + 1, dtype=np.int32)
    vp, f2, vmax, pt = fk.c_pm3_force_kernel(img, isort, np.full(L.ns3, 2, np.int32), ixyz3_table(L), RATIO_SF,
                                             1.0, SIXPI, 1.0)
    G = O.green(L.ng * 2, 4.0, 0.0, 0.5)
    ref = O.pm3_periodic(img, 2, G, 1.0, SIXPI, 1.0)
    act = img.active
    assert _rel_rms((vp - img.vp)[act].astype(np.float64), (ref["vp"] - img.vp)[act].astype(np.float64)) < TOL
    assert np.all(vp[~act] == img.vp[~act])
    assert abs(f2 - ref["f2max"]) <= 1e-5 * ref["f2max"]
    np.testing.assert_allclose(vmax, ref["vmax"], rtol=1e-5)
    assert pt.sum() == act.sum()


@pytest.mark.parametrize("ng", [64, 128])
def test_pm3_periodic_mesh_sides(gpu, ng):
    """Periodic meshes of 128^3 and 256^3 (the k-space step of two-dimensional plane transforms
    around the fused z transforms, all Stockham passes through shared memory) against the
    restatement, on 20 000 uniform particles."""
    from cube2_b200 import ic
    from cube2_b200.kick import CUBE_PM3_PERIODIC, FineKick
    from cube2_b200.layout import RATIO_SF, Layout, build_image, ixyz3_table
    from oracle import oracle as O
    L = Layout(ng=ng, nnt=2, nns=2, ratio_cs=4, ngb=4, app=0.1)
    pos, vel = ic.uniform_random(20000, float(ng), 11)
    img = build_image(pos, vel, L)
    fk = FineKick(L, pm3_mode=CUBE_PM3_PERIODIC, apm3f=4.0)
    vp, f2, vmax, pt = fk.c_pm3_force_kernel(img, np.arange(1, L.ns3 + 1, dtype=np.int32), np.full(L.ns3, 2, np.int32),
                                             ixyz3_table(L), RATIO_SF, 1.0, SIXPI, 1.0)
    ref = O.pm3_periodic(img, 2, O.green(L.ng * 2, 4.0, 0.0, 0.5), 1.0, SIXPI, 1.0)
    act = img.active
    assert _rel_rms((vp - img.vp)[act].astype(np.float64), (ref["vp"] - img.vp)[act].astype(np.float64)) < TOL
    assert abs(f2 - ref["f2max"]) <= 1e-5 * ref["f2max"]
    np.testing.assert_allclose(vmax, ref["vmax"], rtol=1e-5)


def test_pm3_periodic_crowded_brick(gpu):
    """A clump of 12 000 particles inside one brick of 16^3 mesh points (over 2048, so the
    deposit splits the brick into several work items whose windows add up in the mesh), on
    20 000 uniform ones, against the restatement."""
    from cube2_b200 import ic
    from cube2_b200.kick import CUBE_PM3_PERIODIC, FineKick
    from cube2_b200.layout import RATIO_SF, Layout, build_image, ixyz3_table
    from oracle import oracle as O
    L = Layout(ng=64, nnt=2, nns=2, ratio_cs=4, ngb=4, app=0.1)
    pos, vel = ic.uniform_random(20000, 64.0, 12)
    rng = np.random.default_rng(13)
    clump = np.mod(np.array([20.3, 33.7, 41.1]) + 0.8 * rng.standard_normal((12000, 3)), 64.0)
    pos = np.concatenate([pos, clump])
    vel = np.concatenate([vel, (0.05 * rng.standard_normal((12000, 3))).astype(np.float32)])
    brick = np.floor(pos / 8).astype(int)  # 16 mesh points = 8 fine cells at ratio_sf 2
    assert np.bincount((brick[:, 2] * 8 + brick[:, 1]) * 8 + brick[:, 0]).max() > 2048
    img = build_image(pos, vel, L)
    fk = FineKick(L, pm3_mode=CUBE_PM3_PERIODIC, apm3f=4.0)
    vp, f2, vmax, pt = fk.c_pm3_force_kernel(img, np.arange(1, L.ns3 + 1, dtype=np.int32), np.full(L.ns3, 2, np.int32),
                                             ixyz3_table(L), RATIO_SF, 1.0, SIXPI, 1.0)
    ref = O.pm3_periodic(img, 2, O.green(L.ng * 2, 4.0, 0.0, 0.5), 1.0, SIXPI, 1.0)
    act = img.active
    assert _rel_rms((vp - img.vp)[act].astype(np.float64), (ref["vp"] - img.vp)[act].astype(np.float64)) < TOL
    assert abs(f2 - ref["f2max"]) <= 1e-5 * ref["f2max"]
    np.testing.assert_allclose(vmax, ref["vmax"], rtol=1e-5)


@pytest.mark.parametrize("mixed", [False, True])
def test_pm3_subtile_matches_restatement(gpu, mixed):
    """Reference geometry: nft = nfp + 2 nfb meshes per subtile, range-limited Green tables
    (apm3f = 3.5 mesh cells soft, apm2f = 3.5*ratio_sf range, initialize.f90:142-168)."""
    from cube2_b200.kick import CUBE_PM3_SUBTILE, FineKick
    from cube2_b200.layout import RATIO_SF, ixyz3_table
    from oracle import oracle as O
    img, _ = load_golden("t32")
    L = img.layout
    ires = np.full(L.ns3, 2, np.int32)
    if mixed:
        ires[::3] = 3
    greens = {}
    for lev in sorted(set(ires.tolist())):
        rsf = int(RATIO_SF[lev - 1])
        nft = L.ntt * L.ratio_cs * rsf + 2 * L.ratio_cs * rsf
        greens[lev] = O.green(nft, 3.5, 3.5 * rsf, 1.0 / rsf)
    fk = FineKick(L, pm3_mode=CUBE_PM3_SUBTILE)
    isort = np.arange(1, L.ns3 + 1, dtype=np.int32)
    ix = ixyz3_table(L)
    vp, f2, vmax, pt = fk.c_pm3_force_kernel(img, isort, ires, ix, RATIO_SF, 1.0, SIXPI, 1.0, greens=greens)
    ref = O.pm3_subtile(img, ires, ix, RATIO_SF, greens, 1.0, SIXPI, 1.0)
    act = img.active
    assert _rel_rms((vp - img.vp)[act].astype(np.float64), (ref["vp"] - img.vp)[act].astype(np.float64)) < TOL
    assert abs(f2 - ref["f2max"]) <= 1e-5 * ref["f2max"]
    np.testing.assert_allclose(vmax, ref["vmax"], rtol=1e-5)
    assert pt.sum() == act.sum()


def test_pm3_linear_in_mass(gpu):
    """density * mass (kick.f90:463): the PM3 kick is linear in the particle mass."""
    from cube2_b200.kick import FineKick
    from cube2_b200.layout import RATIO_SF, ixyz3_table
    img, _ = load_golden("t32")
    L = img.layout
    fk = FineKick(L)
    isort = np.arange(1, L.ns3 + 1, dtype=np.int32)
    ires = np.full(L.ns3, 2, np.int32)
    z = img.vp * 0
    a = fk.c_pm3_force_kernel(img, isort, ires, ixyz3_table(L), RATIO_SF, 1.0, SIXPI, 1.0, vp=z.copy())[0]
    b = fk.c_pm3_force_kernel(img, isort, ires, ixyz3_table(L), RATIO_SF, 3.0, SIXPI, 1.0, vp=z.copy())[0]
    assert _rel_rms(b.astype(np.float64), 3.0 * a.astype(np.float64)) < 1e-6


@pytest.mark.parametrize("layer", [1, 2])
@pytest.mark.parametrize("ngb", [4, 16])
def test_pm1_pm2_match_restatement(gpu, layer, ngb):
    """PM1 (periodic coarse mesh) and PM2 (per-tile buffered fine mesh) on the GPU against the
    restatement of particle_mesh.f90 / pm_thread with the PM1 and PM2 parameters."""
    from cube2_b200 import ic
    from cube2_b200 import longrange as LR
    from cube2_b200.layout import Layout, build_image
    from oracle import oracle as O
    L = Layout(ng=32, nnt=2, nns=2, ratio_cs=4, ngb=ngb, app=0.1)
    pos, vel = ic.uniform_random(3000, 32.0, 13)
    img = build_image(pos, vel, L)
    if layer == 1:
        vp, f2, vmax = LR.pm1_force(img, 3.5, 1.0, SIXPI, 1.0)
        ref = O.pm1(img, 3.5, 1.0, SIXPI, 1.0)
    else:
        vp, f2, vmax = LR.pm2_force(img, 3.5, 14.0, 1.0, SIXPI, 1.0)
        ref = O.pm2(img, 3.5, 14.0, 1.0, SIXPI, 1.0)
    act = img.active
    assert _rel_rms((vp - img.vp)[act].astype(np.float64), (ref["vp"] - img.vp)[act].astype(np.float64)) < TOL
    assert np.all(vp[~act] == img.vp[~act])
    assert abs(f2 - ref["f2max"]) <= 1e-5 * ref["f2max"]
    np.testing.assert_allclose(vmax, ref["vmax"], rtol=1e-5)
