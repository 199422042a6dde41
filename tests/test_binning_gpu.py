"""PP binning on the GPU is bit-exact with the reference's own arrays (pp_force_kernel.c:196-274)."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

CASES = ["t32", "t32_edge", "t32b_edge"]


def _compare_tile(mine, keys, values, cell_start, xf_sorted, ip_local):
    np.testing.assert_array_equal(mine["keys"], keys)
    np.testing.assert_array_equal(mine["cell_start"], cell_start)
    np.testing.assert_array_equal(mine["ip"], ip_local[values.astype(np.int64)])
    np.testing.assert_array_equal(mine["xf"].view(np.uint32), xf_sorted.view(np.uint32))


@pytest.mark.parametrize("case", CASES)
def test_binning_matches_reference_golden(gpu, case):
    from cube2_b200.kick import FineKick
    from cube2_b200.layout import RATIO_SF, ixyz3_table
    img, z = load_golden(case)
    L = img.layout
    fk = FineKick(L)
    ires = np.full(L.ns3, 2, np.int32)
    ix = ixyz3_table(L)
    for t in range(L.nnt ** 3):
        mine = fk.pp_bin_tile(img, t, ires, ix, RATIO_SF)
        _compare_tile(mine, z[f"t{t}_keys"], z[f"t{t}_values"], z[f"t{t}_cell_start"], z[f"t{t}_xf_sorted"],
                      z[f"t{t}_ip_local"])


def _spread2(v):
    """Bits 0 and 1 of v to bits 0 and 3 (one axis of a 2-bit-per-axis Morton index)."""
    return (v & 1) | ((v & 2) << 2)


@pytest.mark.parametrize("case", CASES)
def test_kick_order_is_a_within_cell_permutation(gpu, case):
    """The kick's spatial order keeps the reference keys and cell_start bit for bit and only
    permutes particles inside each PP cell, into the order of their Morton sub-cell, then
    storage slot (t32_edge's crowded coarse cell of 300 particles also covers the particles
    past the first 128, which the placement pass classifies again)."""
    from cube2_b200.kick import FineKick
    from cube2_b200.layout import RATIO_SF, ixyz3_table
    img, z = load_golden(case)
    L = img.layout
    fk = FineKick(L)
    ires = np.full(L.ns3, 2, np.int32)
    ix = ixyz3_table(L)
    rcp = int(RATIO_SF[1])  # PP cells per coarse cell at level 2; the space order needs 2 or 4
    assert rcp in (2, 4)
    for t in range(L.nnt ** 3):
        ref = fk.pp_bin_tile(img, t, ires, ix, RATIO_SF, spatial=False)
        sp = fk.pp_bin_tile(img, t, ires, ix, RATIO_SF, spatial=True)
        np.testing.assert_array_equal(sp["keys"], z[f"t{t}_keys"])
        np.testing.assert_array_equal(sp["cell_start"], z[f"t{t}_cell_start"])
        cs = sp["cell_start"]
        for c in np.nonzero(np.diff(cs))[0]:
            a, b = cs[c], cs[c + 1]
            assert sorted(sp["ip"][a:b]) == sorted(ref["ip"][a:b])
            # positions travel with their particles
            order_s = np.argsort(sp["ip"][a:b])
            order_r = np.argsort(ref["ip"][a:b])
            np.testing.assert_array_equal(sp["xf"][:, a:b][:, order_s], ref["xf"][:, a:b][:, order_r])
            # inside the cell: Morton index of the 1/8-coarse-cell sub-cell, then storage slot
            x = sp["xf"][:, a:b].astype(np.float64) / L.ratio_cs  # coarse-cell units, exact
            f = np.clip(np.floor(8 * x) - 8 * np.floor(x), 0, 7).astype(np.int64) & (8 // rcp - 1)
            m = _spread2(f[0]) | (_spread2(f[1]) << 1) | (_spread2(f[2]) << 2)
            assert np.all(np.diff(m * (1 << 40) + sp["ip"][a:b]) > 0)


def test_binning_zeldovich_box_matches_reference(gpu):
    """64^3 Zel'dovich lattice (one periodic tile) against the compiled reference, live."""
    from cube2_b200 import ic
    from cube2_b200.kick import FineKick
    from cube2_b200.layout import RATIO_SF, Layout, apm3_table, build_image, ixyz3_table
    from oracle import oracle as O
    from oracle.layouts import LAYOUTS
    L = Layout(**LAYOUTS["cfg0"])
    pos, vel, _ = ic.zeldovich_lattice(64, 0.5, 1000)
    img = build_image(pos, vel, L)
    try:
        ref = O.RefPP(L)
    except FileNotFoundError:
        pytest.skip("reference build not present")
    cap = ref.tile(img, (0, 0, 0), 2, apm3_table(4.0), RATIO_SF, 1.0, 1.0, 1.0, capture=True)
    mine = FineKick(L).pp_bin_tile(img, 0, np.full(L.ns3, 2, np.int32), ixyz3_table(L), RATIO_SF)
    _compare_tile(mine, cap["keys"], cap["values"], cap["cell_start"], cap["xf_sorted"], cap["ip_local"])


def test_binning_float_rounding_spills(gpu):
    """Tiles of 256 coarse cells: (float)(c + (65535.5)/2^16) rounds up to c+1 for c >= 128, so the
    reference key of such a particle lies in the next coarse cell's first PP cell.  The stable order
    (pp_force_kernel.c:244) places it ahead of that cell's own particles; the GPU counting sort must too."""
    from cube2_b200.kick import FineKick
    from cube2_b200.layout import Image, Layout, ixyz3_table
    from oracle.binning import bin_tile
    L = Layout(ng=1024, nnt=1, nns=1, ratio_cs=4, ngb=4, app=0.1)
    rng = np.random.default_rng(9)
    nte = L.nte
    rhoc = np.zeros((1, 1, 1, nte, nte, nte), np.int32)
    cells = []
    # crowd a few cells in the spill range with u = 65535 particles and ordinary ones
    for (i, j, k) in [(130, 5, 5), (131, 5, 5), (200, 140, 7), (150, 150, 150), (3, 3, 3)]:
        m = 6
        rhoc[0, 0, 0, k + 1, j + 1, i + 1] = m
        cells.append(((k + 1, j + 1, i + 1), m))
    order = sorted(cells)
    xp = []
    for (_, m) in order:
        u = rng.integers(0, 65536, size=(m, 3))
        u[: m // 2, rng.integers(0, 3)] = 65535
        xp.append(u.astype(np.uint16).view(np.int16))
    xp = np.concatenate(xp)
    idx = np.cumsum(rhoc.sum(axis=-1).reshape(-1)).reshape(1, 1, 1, nte, nte).astype(np.int64)
    img = Image(L, xp, np.zeros(xp.shape, np.float32), rhoc, idx, np.zeros(xp.shape[0], np.int64),
                np.ones(xp.shape[0], bool), xp.shape[0])
    ratio_sf = np.array([1, 1, 4, 6, 8, 12, 16], np.int32)  # level 2 -> rcp = 1
    want = bin_tile(img, (0, 0, 0), rcp=1)
    # the case really exercises the spill path: some keys lie outside their particle's coarse cell
    S = L.nt + 2
    kx = want["keys"].astype(np.int64) % S
    cell_x = np.repeat([c[0][2] for c in order], [m for _, m in order])[want["values"]]
    assert np.any(kx != cell_x)
    from oracle import oracle as O
    try:
        cap = O.RefPP(L).tile(img, (0, 0, 0), 2, np.full(7, 1.0, np.float32), ratio_sf, 1.0, 1.0, 1.0,
                              capture=True)
        for k in ("keys", "values", "cell_start", "ip_local"):
            np.testing.assert_array_equal(want[k], cap[k])
        np.testing.assert_array_equal(want["xf_sorted"], cap["xf_sorted"])
    except FileNotFoundError:
        pass  # the restatement is pinned against the reference on the golden cases
    mine = FineKick(L).pp_bin_tile(img, 0, np.full(L.ns3, 2, np.int32), ixyz3_table(L), ratio_sf)
    _compare_tile(mine, want["keys"], want["values"], want["cell_start"], want["xf_sorted"], want["ip_local"])
