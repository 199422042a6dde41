"""Batched independent periodic boxes (PM3 geometry CUBE_PM3_TILE_PERIODIC).

A batch of boxes is stored as the parent tiles of one image; each box is its own
periodic box with its own PM3 mesh, and all boxes run in one launch per stage.
The batched kick must equal, box by box, the restatement of the reference PM3 on
that box alone (1e-5 relative rms) and the library's own one-box kick.
"""
import numpy as np
import pytest

SIXPI = np.float32(6 * np.pi)
TOL = 1e-5


def _rel_rms(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def _boxes():
    from cube2_b200 import ic
    from cube2_b200 import workloads as W
    return [ic.zeldovich_box(int(m), 32.0, 0.5, 3100 + t) for t, m in enumerate(W.batch_counts("batch8"))]


def _tables(L):
    from cube2_b200.layout import RATIO_SF, apm3_table, ixyz3_table
    return (np.arange(1, L.ns3 + 1, dtype=np.int32), np.full(L.ns3, 2, np.int32), ixyz3_table(L), apm3_table(4.0),
            RATIO_SF.copy())


def test_batch_layout_matches_one_box_images():
    """The batch image holds every box's own one-tile image, back to back (host only)."""
    from cube2_b200 import workloads as W
    from cube2_b200.layout import build_image, build_tile_batch
    boxes = _boxes()
    tl = W.tile_layout("batch8")
    img = build_tile_batch(boxes, tl, 2)
    off = 0
    for t, (p, v) in enumerate(boxes):
        one = build_image(p, v, tl)
        np.testing.assert_array_equal(img.xp[off:off + one.n_used], one.xp)
        np.testing.assert_array_equal(img.rhoc.reshape(8, -1)[t], one.rhoc.reshape(-1))
        np.testing.assert_array_equal(img.idx_b_r.reshape(8, -1)[t], one.idx_b_r.reshape(-1) + off)
        off += one.n_used
    assert off == img.n_used


@pytest.mark.gpu
def test_pm3_batch_matches_restatement_per_box(gpu):
    from cube2_b200 import workloads as W
    from cube2_b200.kick import CUBE_PM3_TILE_PERIODIC, FineKick
    from cube2_b200.layout import build_image, build_tile_batch
    from oracle import oracle as O
    boxes = _boxes()
    tl = W.tile_layout("batch8")
    img = build_tile_batch(boxes, tl, 2)
    L = img.layout
    isort, ires, ix, _, rs = _tables(L)
    fk = FineKick(L, pm3_mode=CUBE_PM3_TILE_PERIODIC, apm3f=4.0)
    vp, f2, vmax, pt = fk.c_pm3_force_kernel(img, isort, ires, ix, rs, 1.0, SIXPI, 1.0)
    G = O.green(64, 4.0, 0.0, 0.5)
    off, f2ref, vref = 0, 0.0, np.zeros(3)
    for p, v in boxes:
        one = build_image(p, v, tl)
        ref = O.pm3_periodic(one, 2, G, 1.0, SIXPI, 1.0)
        sl = slice(off, off + one.n_used)
        act = one.active
        assert _rel_rms((vp[sl] - one.vp)[act].astype(np.float64), (ref["vp"] - one.vp)[act].astype(np.float64)) < TOL
        assert np.all(vp[sl][~act] == one.vp[~act])
        f2ref = max(f2ref, ref["f2max"])
        vref = np.maximum(vref, ref["vmax"])
        off += one.n_used
    assert abs(f2 - f2ref) <= 1e-5 * f2ref
    np.testing.assert_allclose(vmax, vref, rtol=1e-5)
    assert pt.sum() == img.active.sum()


@pytest.mark.gpu
def test_kick_batch_equals_one_box_kicks(gpu):
    """One batched kick (PM3 + PP over all boxes) against a loop of one-box kicks."""
    from cube2_b200 import workloads as W
    from cube2_b200.kick import CUBE_PM3_PERIODIC, CUBE_PM3_TILE_PERIODIC, FineKick
    from cube2_b200.layout import build_image, build_tile_batch
    boxes = _boxes()
    tl = W.tile_layout("batch8")
    img = build_tile_batch(boxes, tl, 2)
    isort, ires, ix, apm3, rs = _tables(img.layout)
    vb, outb = FineKick(img.layout, pm3_mode=CUBE_PM3_TILE_PERIODIC, apm3f=4.0).kick_fine(
        img, isort, ires, ix, apm3, rs, 1.0, SIXPI, 1.0)
    fk1 = FineKick(tl, pm3_mode=CUBE_PM3_PERIODIC, apm3f=4.0)
    t1 = _tables(tl)
    off, f2 = 0, 0.0
    for p, v in boxes:
        one = build_image(p, v, tl)
        v1, o1 = fk1.kick_fine(one, *t1, 1.0, SIXPI, 1.0)
        sl = slice(off, off + one.n_used)
        assert _rel_rms((vb[sl] - one.vp).astype(np.float64), (v1 - one.vp).astype(np.float64)) < TOL
        f2 = max(f2, o1[1])
        off += one.n_used
    assert abs(outb[1] - f2) <= 1e-5 * f2
