"""Host-side data formats: the reference particle layout, subtile tables and classification."""
import numpy as np
import pytest

from cube2_b200 import ic
from cube2_b200.layout import (Layout, build_image, classify_subtiles, decode_positions, encode_positions,
                               indexed_sort, ixyz3_table)


@pytest.mark.parametrize("nnt,ngb", [(1, 4), (2, 4), (2, 8)])
def test_build_image_layout_invariants(nnt, ngb):
    L = Layout(ng=32, nnt=nnt, nns=2, ratio_cs=4, ngb=ngb, app=0.1)
    pos, vel = ic.uniform_random(3000, 32.0, 1)
    img = build_image(pos, vel, L)
    nt, ncb, nte = L.nt, L.ncb, L.nte
    # every physical particle appears exactly once as an interior copy
    assert img.active.sum() == 3000
    assert np.array_equal(np.sort(img.pid[img.active]), np.arange(3000))
    # spine: idx_b_r is the running row count (variables.f90:146-216)
    rows = img.rhoc.sum(axis=-1).reshape(-1)
    assert np.array_equal(np.cumsum(rows), img.idx_b_r.reshape(-1))
    assert img.idx_b_r.reshape(-1)[-1] == img.n_used
    # decode of every stored copy lands in its cell and reproduces the encoded position (mod box)
    cc, u = encode_positions(pos, L.ratio_cs, L.nc)
    flat = img.rhoc.reshape(-1)
    start = np.cumsum(flat) - flat
    tt = np.arange(L.nnt)
    e = np.arange(nte) - ncb
    tz, ty, tx, k, j, i = np.meshgrid(tt, tt, tt, e, e, e, indexing="ij")
    cell_of = np.repeat(np.arange(flat.size), flat)
    gxyz = np.stack([(tx * nt + i).reshape(-1), (ty * nt + j).reshape(-1), (tz * nt + k).reshape(-1)], -1)
    g = gxyz[cell_of]
    x = decode_positions(g, img.xp) * L.ratio_cs
    want = (cc[img.pid] + (u[img.pid].astype(np.float64) + 0.5) / 65536.0) * L.ratio_cs
    dx = np.mod(x - want + L.ng / 2, L.ng) - L.ng / 2
    assert np.max(np.abs(dx)) < 1e-9
    assert start[-1] + flat[-1] == img.n_used


def test_fixed_point_round_trip():
    """kick.f90:292 decode of ic.f90:603 encode: |x - decode(encode(x))| <= 2^-17 coarse cells."""
    rng = np.random.default_rng(2)
    pos = rng.random((10000, 3)) * 64
    cc, u = encode_positions(pos, 4, 16)
    xp = u.view(np.int16)
    back = decode_positions(cc, xp) * 4
    assert np.max(np.abs(back - pos)) <= 4 * 2.0 ** -17 + 1e-12
    # u = (uint16)xp: the int16 storage covers the full unsigned range
    assert xp.dtype == np.int16 and u.max() > 32767


def test_ixyz3_order():
    L = Layout(ng=64, nnt=2, nns=2)
    t = ixyz3_table(L)
    assert t.shape == (64, 6)
    assert list(t[0]) == [1, 1, 1, 1, 1, 1] and list(t[1]) == [2, 1, 1, 1, 1, 1]
    assert list(t[8]) == [1, 1, 1, 2, 1, 1]
    assert list(t[-1]) == [2, 2, 2, 2, 2, 2]


def test_indexed_sort_is_ascending_permutation():
    rng = np.random.default_rng(4)
    for n in (1, 2, 7, 64, 257):
        a = rng.standard_normal(n).astype(np.float32)
        idx = indexed_sort(a)
        assert sorted(idx.tolist()) == list(range(1, n + 1))
        assert np.all(np.diff(a[idx - 1]) >= 0)


def test_classify_thresholds():
    """kick.f90:114-127: npc_max = max(rhoc)/64 against 24 / 114 / 320 / 1350."""
    L = Layout(ng=32, nnt=1, nns=2, ratio_cs=4, ngb=4)
    rhoc = np.zeros((1, 1, 1, L.nte, L.nte, L.nte), np.int32)
    peaks = [24 * 64 - 1, 24 * 64, 114 * 64, 1350 * 64, 10, 320 * 64, 0, 200 * 64]
    want = [2, 3, 4, 6, 2, 5, 2, 4]
    for s in range(8):
        sx, sy, sz = s % 2, (s // 2) % 2, s // 4
        rhoc[0, 0, 0, 1 + sz * 4, 1 + sy * 4, 1 + sx * 4] = peaks[s]
    ires, isort = classify_subtiles(rhoc, L)
    assert list(ires) == want
    # heaviest subtile first (kick.f90:131 sorts -npc_max ascending)
    assert isort[0] == 4
