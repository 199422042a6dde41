"""PP force and kick on the GPU against the reference CPU kernel (pp_force_kernel.c:282-364).

Forces agree within 1e-5 relative rms (FP32 pair force; the GPU accumulates with
Kahan compensation, the reference in plain FP32 with a different order).
a_mid*dt = 6*pi makes the velocity change equal to the force.
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

SIXPI = np.float32(6 * np.pi)
TOL = 1e-5


def _rel_rms(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def _run_pp(img, fk, ires_value=2, apm3f=4.0, mass=1.0):
    from cube2_b200.layout import RATIO_SF, apm3_table, ixyz3_table
    L = img.layout
    isort = np.arange(1, L.ns3 + 1, dtype=np.int32)
    return fk.c_pp_force_kernel(img, isort, np.full(L.ns3, ires_value, np.int32), ixyz3_table(L),
                                apm3_table(apm3f), RATIO_SF, mass, SIXPI, 1.0)


@pytest.mark.parametrize("case", ["t32", "t32_edge", "t32b_edge"])
def test_pp_matches_reference_golden(gpu, case):
    from cube2_b200.kick import FineKick
    img, z = load_golden(case)
    L = img.layout
    vp, f2, vmax, pt, tt = _run_pp(img, FineKick(L))
    dv = (vp - img.vp).astype(np.float64)
    dref = (z["vp_ref"] - img.vp).astype(np.float64)
    assert _rel_rms(dv, dref) < TOL
    # only interior particles are kicked (pp_force_kernel.c:339-364)
    assert np.all(vp[~img.active] == img.vp[~img.active])
    assert abs(f2 - float(z["f2max_ref"])) <= TOL * float(z["f2max_ref"])
    np.testing.assert_allclose(vmax, z["vmax_ref"], rtol=TOL)
    # ptotal per subtile sums to the reference's per-tile counts
    per_tile = pt.reshape(L.nnt ** 3, L.nns ** 3).sum(axis=1)
    assert per_tile.sum() == z["ptotal_ref"].sum() == img.active.sum()
    assert np.all(tt >= 0)


def test_pp_zeldovich_box_vs_reference_live(gpu):
    """64^3 Zel'dovich lattice (the CPU-runnable workload) against the reference kernel."""
    from cube2_b200 import ic
    from cube2_b200.kick import FineKick
    from cube2_b200.layout import RATIO_SF, Layout, apm3_table, build_image
    from oracle import oracle as O
    from oracle.layouts import LAYOUTS
    L = Layout(**LAYOUTS["cfg0"])
    pos, vel, _ = ic.zeldovich_lattice(64, 0.5, 1000)
    img = build_image(pos, vel, L)
    try:
        ref = O.RefPP(L)
    except FileNotFoundError:
        pytest.skip("reference build not present")
    vref, f2r, vmr, ptr = ref.kick(img, [2], apm3_table(4.0), RATIO_SF, 1.0, SIXPI, 1.0)
    vp, f2, vmax, pt, _ = _run_pp(img, FineKick(L))
    assert _rel_rms((vp - img.vp).astype(np.float64), (vref - img.vp).astype(np.float64)) < TOL
    assert abs(f2 - f2r) <= TOL * f2r
    np.testing.assert_allclose(vmax, vmr, rtol=TOL)
    assert pt.sum() == ptr.sum()


def test_pp_mass_and_kick_scaling(gpu):
    """af*mass^2 and dv = af*a_mid*dt/(6 pi) (pp_force_kernel.c:350-357): linear in both."""
    from cube2_b200.kick import FineKick
    from cube2_b200.layout import RATIO_SF, apm3_table, ixyz3_table
    img, _ = load_golden("t32")
    L = img.layout
    fk = FineKick(L)
    isort = np.arange(1, L.ns3 + 1, dtype=np.int32)
    ires = np.full(L.ns3, 2, np.int32)
    zero_v = img.vp * 0
    v1, f1, _, _, _ = fk.c_pp_force_kernel(img, isort, ires, ixyz3_table(L), apm3_table(4.0), RATIO_SF, 1.0,
                                           SIXPI, 1.0, vp=zero_v.copy())
    v2, f2, _, _, _ = fk.c_pp_force_kernel(img, isort, ires, ixyz3_table(L), apm3_table(4.0), RATIO_SF, 2.0,
                                           SIXPI, 0.5, vp=zero_v.copy())
    np.testing.assert_allclose(v2, v1 * 2.0, rtol=1e-6, atol=1e-6)
    assert abs(f2 - 16.0 * f1) <= 1e-5 * 16 * f1


def test_pp_repeatable(gpu):
    """Deterministic: the persistent queue changes order, not the arithmetic of any particle."""
    from cube2_b200.kick import FineKick
    img, _ = load_golden("t32_edge")
    fk = FineKick(img.layout)
    a = _run_pp(img, fk)[0]
    b = _run_pp(img, fk)[0]
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("levels", [(2, 3), (3, 4), (2, 6)])
def test_pp_mixed_levels_in_one_tile(gpu, levels):
    """Subtiles of one parent tile at different levels: the tile's PP grid takes the finest
    ratio_sf, and every particle keeps the range of its own subtile, so a particle of the
    coarser level searches R = ceil(rc*rcp/ratio_cs) > 1 cells (pp_force_kernel.cu:205)."""
    from cube2_b200 import ic
    from cube2_b200.kick import FineKick
    from cube2_b200.layout import RATIO_SF, Layout, apm3_table, build_image, encode_positions, ixyz3_table
    from oracle.pp_direct import pp_forces
    L = Layout(ng=32, nnt=2, nns=2, ratio_cs=4, ngb=4, app=0.1)
    pos, vel = ic.uniform_random(12000, 32.0, 31)
    img = build_image(pos, vel, L)
    ix = ixyz3_table(L)
    ires = np.array([levels[(k % 3) == 0] for k in range(L.ns3)], np.int32)
    apm3 = apm3_table(3.5)
    vp, _, _, _, _ = FineKick(L).c_pp_force_kernel(img, np.arange(1, L.ns3 + 1, dtype=np.int32), ires, ix, apm3,
                                                   RATIO_SF, 1.0, SIXPI, 1.0, vp=np.zeros_like(img.vp))
    # range of each physical particle from its subtile
    cc, u = encode_positions(pos, 4, 8)
    posq = (cc + (u.astype(np.float64) + 0.5) / 65536.0) * 4.0
    tx, ty, tz = cc[:, 0] // L.nt, cc[:, 1] // L.nt, cc[:, 2] // L.nt
    sx, sy, sz = (cc[:, 0] % L.nt) // L.ntt, (cc[:, 1] % L.nt) // L.ntt, (cc[:, 2] % L.nt) // L.ntt
    loc = (((tz * 2 + ty) * 2 + tx) * 2 + sz) * 4 + sy * 2 + sx
    it_of_loc = np.zeros(L.ns3, np.int64)
    for it, r in enumerate(ix):
        it_of_loc[(((r[5] - 1) * 2 + r[4] - 1) * 2 + r[3] - 1) * 8 + (r[2] - 1) * 4 + (r[1] - 1) * 2 + r[0] - 1] = it
    ranges = apm3[ires[it_of_loc[loc]] - 1].astype(np.float64)
    F = pp_forces(posq, 32.0, 0.1, ranges)
    kick = float(np.float32(SIXPI) / np.float32(6.0)) / np.pi
    mine = np.zeros_like(F)
    act = img.active
    mine[img.pid[act]] = vp[act].astype(np.float64) / kick
    assert _rel_rms(mine, F) < TOL


def test_pair_count_matches_kdtree(gpu):
    """The algorithmic work counter: ordered pairs 0 < r < 2 in the periodic box (scipy cKDTree)."""
    from scipy.spatial import cKDTree
    from cube2_b200 import ic
    from cube2_b200.kick import FineKick
    from cube2_b200.layout import RATIO_SF, Layout, apm3_table, build_image, encode_positions, ixyz3_table
    L = Layout(ng=32, nnt=2, nns=2, ratio_cs=4, ngb=4, app=0.1)
    pos, vel = ic.uniform_random(20000, 32.0, 21)
    img = build_image(pos, vel, L)
    n = FineKick(L).pp_pair_count(img, np.full(L.ns3, 2, np.int32), ixyz3_table(L), apm3_table(4.0), RATIO_SF)
    cc, u = encode_positions(pos, 4, 8)
    posq = np.mod((cc + (u.astype(np.float64) + 0.5) / 65536.0) * 4.0, 32.0)
    tree = cKDTree(posq, boxsize=32.0)
    want = tree.count_neighbors(tree, 2.0 * (1 - 1e-7)) - len(posq)
    assert abs(n - want) <= 2e-6 * want + 2, (n, want)


def test_pp_empty_image(gpu):
    from cube2_b200.kick import FineKick
    from cube2_b200.layout import Image, Layout
    L = Layout(ng=32, nnt=2, nns=2, ratio_cs=4, ngb=4, app=0.1)
    img = Image(L, np.zeros((0, 3), np.int16), np.zeros((0, 3), np.float32),
                np.zeros((2, 2, 2, L.nte, L.nte, L.nte), np.int32), np.zeros((2, 2, 2, L.nte, L.nte), np.int64),
                np.zeros(0, np.int64), np.zeros(0, bool), 0)
    vp, f2, vmax, pt, _ = _run_pp(img, FineKick(L))
    assert f2 == 0.0 and np.all(vmax == 0) and pt.sum() == 0
