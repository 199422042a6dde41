"""PP on clustered boxes against the reference's own CPU PP kernel (pp_force_kernel.c:282-364).

Lognormal (sigma_lnrho = 1.5) Poisson samples put hundreds of particles in some fine
cells, so the kick's work list splits crowded PP cells into several chunk items and
groups sparse neighbouring cells along x (csrc/pp.cu).  The test asserts that both paths
are reached (cube_pp_work_stats), under the autotuned shape and under the shapes with the
smallest and the largest chunk, and that every one gives the reference's kick within 1e-5
relative rms, with f2max and vmax within 1e-5.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIXPI = float(np.float32(6 * np.pi))
TOL = 1e-5

_CASES = {}


def _case(name):
    if name not in _CASES:
        from cube2_b200 import ic
        from cube2_b200.layout import Layout, build_image
        from oracle import oracle as O
        from oracle.layouts import LAYOUTS
        if name == "clumpy64":
            L = Layout(**LAYOUTS["cfg0"])
            pos, vel, counts = ic.lognormal_poisson(64, 1.5, 4100)
        else:
            L = Layout(**LAYOUTS["c96"])
            pos, vel, counts = ic.lognormal_poisson(96, 1.5, 4200)
        img = build_image(pos, vel, L)
        from cube2_b200.layout import RATIO_SF, apm3_table
        apm3 = apm3_table(4.0)
        ref = O.RefPP(L).kick(img, [2] * L.nnt ** 3, apm3, RATIO_SF, 1.0, SIXPI, 1.0)
        _CASES[name] = (img, int(counts.max()), ref)
    return _CASES[name]


def _shape_index(which):
    from cube2_b200 import kick as K
    table, _ = K.pp_shapes()
    if which == "autotune":
        return -1
    chunks = [t["chunk"] for t in table]
    c = min(chunks) if which == "smallest_chunk" else max(chunks)
    return chunks.index(c)


@pytest.mark.parametrize("name", ["clumpy64", "clumpy96"])
@pytest.mark.parametrize("which", ["autotune", "smallest_chunk", "largest_chunk"])
def test_clustered_pp_matches_reference(gpu, name, which):
    from cube2_b200 import kick as K
    from cube2_b200.layout import RATIO_SF, apm3_table, ixyz3_table
    img, max_occ, (vref, f2ref, vmaxref, _) = _case(name)
    L = img.layout
    assert max_occ >= 100  # crowded fine cells
    fk = K.FineKick(L, pm3_mode=K.CUBE_PM3_PERIODIC, apm3f=4.0)
    k = _shape_index(which)
    try:
        K.pp_set_shape(k)
        vp, f2, vmax, pt, _ = fk.c_pp_force_kernel(img, np.arange(1, L.ns3 + 1, dtype=np.int32),
                                                   np.full(L.ns3, 2, np.int32), ixyz3_table(L), apm3_table(4.0),
                                                   RATIO_SF, 1.0, SIXPI, 1.0)
        stats = K.pp_work_stats()
        chunk = K.pp_shapes()[0][K.pp_shapes()[1]]["chunk"]
    finally:
        K.pp_set_shape(-1)
    act = img.active
    dv = (vp - img.vp).astype(np.float64)[act]
    dref = (vref - img.vp).astype(np.float64)[act]
    err = float(np.sqrt(np.sum((dv - dref) ** 2) / np.sum(dref ** 2)))
    assert err < TOL, (which, err)
    assert abs(f2 - f2ref) <= TOL * f2ref
    np.testing.assert_allclose(vmax, vmaxref, rtol=TOL)
    assert pt.sum() == act.sum()
    # the work list reached chunk splitting and sparse-cell grouping
    assert stats["split_items"] > 0 and stats["grouped_items"] > 0, stats
    assert stats["max_ni"] == chunk, (stats, chunk)
    assert stats["items"] > stats["split_items"] > 0
