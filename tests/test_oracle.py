"""The CPU oracle pinned against the reference's golden vectors and against physics truth."""
import os

import numpy as np
import pytest

from conftest import HERE, load_golden

GOLD = os.path.join(HERE, "golden")
CASES = ["t32", "t32_edge", "t32b_edge"]


def _ref_available(layout):
    from oracle import oracle as O
    try:
        O.RefPP(layout)
        return True
    except FileNotFoundError:
        return False


def test_fra_oracle_matches_reference_golden(oracle_lib):
    """FP64 F_ra restatement (oracle/ewald.c) vs the reference's F_ra values (pp_force_kernel.c:45-74)."""
    from oracle import oracle as O
    z = np.load(os.path.join(GOLD, "fra.npz"))
    for a_i, apm in enumerate(z["apm"]):
        ref = z["F"][a_i].astype(np.float64)
        mine = np.array([O.F_ra64(float(r), float(apm)) for r in z["r"]])
        rel = np.abs(mine - ref) / np.maximum(np.abs(ref), 1e-30)
        # single-precision reference vs double restatement
        assert np.max(rel[np.abs(ref) > 1e-3]) < 2e-4, (apm, np.max(rel))


@pytest.mark.parametrize("n", [16, 20, 24])
def test_green_restatement_golden(oracle_lib, n):
    from oracle import oracle as O
    z = np.load(os.path.join(GOLD, f"green_{n}.npz"))
    G = O.green(int(z["n"]), float(z["apm_soft"]), float(z["apm_range"]), float(z["gridsize"]))
    np.testing.assert_array_equal(G, z["G"])
    # Gk(::n/2,::n/2,::n/2) = 0 (Green.f90:71) and G even in every axis
    h = n // 2
    for a in (0, h):
        for b in (0, h):
            for c in (0, h):
                assert G[c, b, a] == 0.0
    np.testing.assert_allclose(G[1:, :, :], G[1:, :, :][::-1], rtol=1e-6, atol=0)


@pytest.mark.parametrize("case", CASES)
def test_binning_restatement_matches_reference_arrays(case):
    """numpy restatement of pp_force_kernel.c:196-274 == the reference's internal arrays, bit for bit."""
    from oracle.binning import bin_tile
    img, z = load_golden(case)
    L = img.layout
    for tz in range(L.nnt):
        for ty in range(L.nnt):
            for tx in range(L.nnt):
                t = (tz * L.nnt + ty) * L.nnt + tx
                mine = bin_tile(img, (tx, ty, tz), rcp=2)
                np.testing.assert_array_equal(mine["keys"], z[f"t{t}_keys"])
                np.testing.assert_array_equal(mine["values"], z[f"t{t}_values"])
                np.testing.assert_array_equal(mine["cell_start"], z[f"t{t}_cell_start"])
                np.testing.assert_array_equal(mine["ip_local"], z[f"t{t}_ip_local"])
                np.testing.assert_array_equal(mine["xf_sorted"].view(np.uint32), z[f"t{t}_xf_sorted"].view(np.uint32))


@pytest.mark.parametrize("case", CASES)
def test_reference_build_reproduces_golden(case):
    """The compiled reference (oracle/_ref) still produces the committed vectors."""
    from cube2_b200.layout import RATIO_SF, apm3_table
    from oracle import oracle as O
    img, z = load_golden(case)
    if not _ref_available(img.layout):
        pytest.skip("reference build not present")
    ref = O.RefPP(img.layout)
    vp, f2, vmax, pt = ref.kick(img, [2] * img.layout.nnt ** 3, apm3_table(4.0), RATIO_SF, 1.0,
                                np.float32(6 * np.pi), 1.0)
    np.testing.assert_array_equal(vp, z["vp_ref"])
    assert f2 == float(z["f2max_ref"])
    np.testing.assert_array_equal(vmax, z["vmax_ref"])
    np.testing.assert_array_equal(pt, z["ptotal_ref"])


def test_ewald_oracle_properties(oracle_lib):
    """FP64 truth: independent of the Ewald split, and pairwise forces cancel."""
    from oracle import oracle as O
    rng = np.random.default_rng(3)
    box = 8.0
    pos = rng.random((300, 3)) * box
    tg = np.arange(300)
    F1 = O.ewald(pos, box, 0.1, tg, alpha=np.sqrt(-np.log(1e-12)) / (0.5 * box), tol=1e-12)
    F2 = O.ewald(pos, box, 0.1, tg, alpha=1.3 * np.sqrt(-np.log(1e-12)) / (0.5 * box), tol=1e-12)
    scale = np.sqrt(np.mean(F1 ** 2))
    assert np.max(np.abs(F1 - F2)) / scale < 1e-6
    # Newton's third law over the whole periodic system
    assert np.max(np.abs(F1.sum(axis=0))) / (scale * 300) < 1e-8


def test_ewald_close_pair_is_softened_newton(oracle_lib):
    """A close pair in a big box: force = F_ra(r, app) (basic_functions.f08:95-109) up to image terms."""
    from oracle import oracle as O
    box = 64.0
    for r in (0.05, 0.3, 1.0):
        pos = np.array([[10.0, 10.0, 10.0], [10.0 + r, 10.0, 10.0]])
        F = O.ewald(pos, box, 0.1, np.array([0]))
        assert abs(F[0, 0] - O.F_ra64(r, 0.1)) / O.F_ra64(r, 0.1) < 1e-4
        assert abs(F[0, 1]) < 1e-8 and abs(F[0, 2]) < 1e-8


def test_pm3_pp_oracle_matches_fp64_truth(oracle_lib):
    """Oracle PM3 (periodic mesh, TSC, Green_3D) + reference PP reproduce the FP64 truth (< 1% rms)."""
    from cube2_b200 import ic
    from cube2_b200.layout import RATIO_SF, Layout, apm3_table, build_image, encode_positions
    from oracle import oracle as O
    L = Layout(ng=32, nnt=2, nns=2, ratio_cs=4, ngb=4, app=0.1)
    if not _ref_available(L):
        pytest.skip("reference build not present")
    pos, vel = ic.uniform_random(32 ** 3 // 4, 32.0, 5)
    img = build_image(pos, vel, L)
    sixpi = np.float32(6 * np.pi)
    vp_pp, _, _, _ = O.RefPP(L).kick(img, [2] * 8, apm3_table(4.0), RATIO_SF, 1.0, sixpi, 1.0)
    G = O.green(64, 4.0, 0.0, 0.5)
    pm = O.pm3_periodic(img, 2, G, 1.0, sixpi, 1.0)
    tot = (vp_pp - img.vp).astype(np.float64) + pm["dv"]
    cc, u = encode_positions(pos, 4, 8)
    posq = (cc + (u.astype(np.float64) + 0.5) / 65536.0) * 4.0
    act = np.nonzero(img.active)[0]
    samp = np.random.default_rng(0).choice(act, 400, replace=False)
    F = O.ewald(posq, 32.0, 0.1, img.pid[samp])
    err = np.sqrt(np.sum((tot[samp] - F) ** 2) / np.sum(F ** 2))
    assert err < 0.01, err


def test_four_layer_split_oracle_matches_fp64_truth(oracle_lib):
    """The reference's whole force split restated: PM1 on the coarse periodic mesh
    (Green_3D(nc, 3.5, 0, ratio_cs)), PM2 on the tile's buffered fine mesh (softening 3.5,
    range 14 fine cells), PM3 on the buffered subtile meshes (3.5 mesh cells soft, range
    apm2f) and PP within 1.75 fine cells sum to the FP64 periodic truth (initialize.f90:129-145,
    parameters.f90:34-40 with ratio_sf = 2)."""
    from cube2_b200 import ic
    from cube2_b200.layout import RATIO_SF, Layout, build_image, encode_positions, ixyz3_table
    from oracle import oracle as O
    from oracle import pp_direct as P
    L = Layout(ng=32, nnt=1, nns=2, ratio_cs=4, ngb=16, app=0.1)
    pos, vel = ic.uniform_random(2048, 32.0, 11)
    img = build_image(pos, vel, L)
    sixpi = np.float32(6 * np.pi)
    p1 = O.pm1(img, 3.5, 1.0, sixpi, 1.0)
    p2 = O.pm2(img, 3.5, 14.0, 1.0, sixpi, 1.0)
    ires = np.full(L.ns3, 2, np.int32)
    nft = L.ntt * L.ratio_cs * 2 + 2 * L.ratio_cs * 2
    p3 = O.pm3_subtile(img, ires, ixyz3_table(L), RATIO_SF, {2: O.green(nft, 3.5, 7.0, 0.5)}, 1.0, sixpi, 1.0)
    cc, u = encode_positions(pos, 4, 8)
    posq = (cc + (u.astype(np.float64) + 0.5) / 65536.0) * 4.0
    pp = P.pp_forces(posq, 32.0, 0.1, np.full(posq.shape[0], 1.75))
    act = np.nonzero(img.active)[0]
    tot = p1["dv"][act] + p2["dv"][act] + p3["dv"][act] + pp[img.pid[act]]
    F = O.ewald(posq, 32.0, 0.1, img.pid[act])

    def err(x):
        return np.sqrt(np.sum((x - F) ** 2) / np.sum(F ** 2))
    assert err(tot) < 0.01, err(tot)  # measured 0.4 %
    # each long-range layer is needed: without it the error is several per cent
    assert err(tot - p1["dv"][act]) > 0.02
    assert err(tot - p2["dv"][act]) > 0.02


def test_reference_cuda_builds_load_and_size_like_the_reference():
    """The reference's CUDA path, built per layout for sm_100a (oracle/build_ref.py), loads
    without a GPU and exports its C ABI (pm3_fft_cuda.cu:516-628, pp_force_kernel.cu:496-547,
    :960); the capacity guard that keeps it from exit()ing uses the reference's own arithmetic
    (pp_force_kernel.cu:45-51)."""
    from oracle import oracle as O
    from oracle.layouts import GPU_BUILDS
    for name, p in GPU_BUILDS.items():
        try:
            r = O.RefCuda(name)
        except FileNotFoundError:
            pytest.skip("reference CUDA build missing (needs the reference tree)")
        for sym in ("c_pm3_force_kernel", "c_pp_force_kernel", "c_gpu_velocity_get", "c_gpu_velocity_finalize",
                    "c_pm3_fft_finalize", "c_select_gpu_for_image"):
            getattr(r.lib, sym)
        nc = p["ng"] // p["ratio_cs"]
        nt = nc // p["nnt"]
        nte = nt + 2 * (p["ngb"] // p["ratio_cs"])
        assert r.np_image_max == int(p["ng"] ** 3 * (nte / nt) ** 3 * p["image_buffer"] + 1e-6)
        assert r.np_tile_max >= p["ng"] ** 3 // p["nnt"] ** 3
