"""Host-side builders of the benchmark's inputs (CPU): the batch of independent periodic boxes
stored as the parent tiles of one image, decoded positions, and the seeded generators."""
import numpy as np

from cube2_b200 import ic
from cube2_b200 import workloads as W
from cube2_b200.layout import Layout, build_image, build_tile_batch


def test_physical_positions_round_trip():
    """The stored fixed-point positions of the physical particles decode to the inputs within
    the fixed-point resolution (ratio_cs / 2^16 fine cells, rounded to the nearest half step)."""
    L = Layout(ng=32, nnt=2, nns=2, ratio_cs=4, ngb=4, app=0.1)
    pos, vel = ic.uniform_random(4000, 32.0, 21)
    img = build_image(pos, vel, L)
    got = W.physical_positions(img)
    d = np.abs(got - pos)
    d = np.minimum(d, 32.0 - d)  # periodic
    assert d.max() <= L.ratio_cs / 65536.0
    # every physical particle is stored exactly once, with its own velocity
    assert img.active.sum() == len(pos)
    np.testing.assert_array_equal(np.sort(img.pid[img.active]), np.arange(len(pos)))
    np.testing.assert_array_equal(img.vp[img.active], vel[img.pid[img.active]])


def test_tile_batch_stores_each_box_as_its_own_periodic_tile():
    """build_tile_batch: tile t holds box t with its own periodic copies (the one-tile image of
    the box), the spine runs over the whole batch, pid numbers box t after boxes 0..t-1, and
    the physical particles decode to the box's positions plus the tile's origin."""
    tile = Layout(ng=16, nnt=1, nns=2, ratio_cs=4, ngb=4, app=0.1)
    nnt = 2
    boxes = [ic.zeldovich_box(m, 16.0, 0.3, 500 + t) for t, m in enumerate([2, 3, 4, 5, 3, 6, 4, 2])]
    img = build_tile_batch(boxes, tile, nnt)
    L = img.layout
    assert (L.ng, L.nnt, L.nt) == (32, 2, tile.nt)
    nte = tile.nte
    assert img.rhoc.shape == (nnt, nnt, nnt, nte, nte, nte)
    starts = np.concatenate([[0], img.idx_b_r.reshape(-1)])
    assert np.all(np.diff(starts) >= 0) and starts[-1] == img.n_used == len(img.xp)
    off_stored, off_pid = 0, 0
    got = W.physical_positions(img)
    for t, (p, v) in enumerate(boxes):
        one = build_image(p, v, tile)
        tz, ty, tx = t // (nnt * nnt), (t // nnt) % nnt, t % nnt
        np.testing.assert_array_equal(img.rhoc[tz, ty, tx], one.rhoc.reshape(nte, nte, nte))
        sl = slice(off_stored, off_stored + one.n_used)
        np.testing.assert_array_equal(img.xp[sl], one.xp)
        np.testing.assert_array_equal(img.vp[sl], one.vp)
        np.testing.assert_array_equal(img.active[sl], one.active)
        np.testing.assert_array_equal(img.pid[sl], one.pid + off_pid)
        # positions: the box's own, shifted to the tile's place in the image
        mine = got[off_pid:off_pid + len(p)] - np.array([tx, ty, tz]) * tile.ng
        d = np.abs(mine - p)
        d = np.minimum(d, tile.ng - d)
        assert d.max() <= tile.ratio_cs / 65536.0
        off_stored += one.n_used
        off_pid += len(p)
    assert img.n_particles == off_pid


def test_lognormal_poisson_is_seeded_and_has_the_requested_mean():
    a = ic.lognormal_poisson(24, 1.5, 7)
    b = ic.lognormal_poisson(24, 1.5, 7)
    c = ic.lognormal_poisson(24, 1.5, 8)
    np.testing.assert_array_equal(a[0], b[0])
    assert not np.array_equal(a[2], c[2])
    pos, _, counts = a
    n3 = 24 ** 3
    assert counts.sum() == len(pos)
    assert abs(len(pos) - n3) < 5 * np.sqrt(n3) + 0.02 * n3  # mean one particle per cell
    assert pos.min() >= 0.0 and pos.max() < 24.0
    # clustered: the occupancy spread is far beyond Poisson's (variance = mean)
    assert counts.var() > 3 * counts.mean()
    # every particle lies in the cell it was counted in
    cell = np.floor(pos).astype(np.int64)
    np.testing.assert_array_equal(np.bincount((cell[:, 2] * 24 + cell[:, 1]) * 24 + cell[:, 0], minlength=n3),
                                  counts.reshape(-1))


def test_batch_counts_are_seeded_cubes_within_the_clip():
    w = W.WORKLOADS["batch512"]
    m = W.batch_counts("batch512")
    assert m.shape == (w["layout"]["nnt"] ** 3,)
    np.testing.assert_array_equal(m, W.batch_counts("batch512"))
    lo, hi = w["clip"]
    # the nearest cube to a count within the clip
    assert (m ** 3).min() >= round(np.cbrt(lo)) ** 3 and (m ** 3).max() <= round(np.cbrt(hi)) ** 3
    assert len(np.unique(m)) > 5  # uneven boxes
