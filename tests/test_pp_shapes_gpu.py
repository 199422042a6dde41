"""PP kernel shapes and their autotuner (cube_pp_set_shape / cube_pp_shapes).

Every shape of the PP force kernel must give the kick of the default shape up to FP32
summation order, on a clustered box whose crowded PP cells are split into several work
items; the autotuner must time every shape once per key, pick the fastest, and keep it
for later kicks with the same key.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIXPI = float(np.float32(6 * np.pi))


def _rel_rms(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


@pytest.fixture(scope="module")
def clumpy():
    from cube2_b200 import ic
    from cube2_b200.layout import RATIO_SF, Layout, apm3_table, build_image, ixyz3_table
    L = Layout(ng=64, nnt=1, nns=2, ratio_cs=4, ngb=4, app=0.1)
    img = build_image(*ic.lognormal_poisson(64, 1.5, 4100)[:2], L)
    tabs = (np.arange(1, L.ns3 + 1, dtype=np.int32), np.full(L.ns3, 2, np.int32), ixyz3_table(L),
            apm3_table(4.0), RATIO_SF.copy())
    return img, tabs


def test_every_shape_gives_the_default_kick(gpu, clumpy):
    from cube2_b200 import kick as K
    img, tabs = clumpy
    fk = K.FineKick(img.layout, pm3_mode=K.CUBE_PM3_PERIODIC)
    table, _ = K.pp_shapes()
    assert len(table) >= 8 and {t["chunk"] for t in table} >= {8, 16, 32}
    try:
        K.pp_set_shape(0)
        want, f2_want, vmax_want, _, _ = fk.c_pp_force_kernel(img, *tabs, 1.0, SIXPI, 1.0)
        dv_want = (want - img.vp).astype(np.float64)
        assert np.sum(dv_want[img.active] ** 2) > 0
        for k in range(1, len(table)):
            K.pp_set_shape(k)
            got, f2, vmax, _, _ = fk.c_pp_force_kernel(img, *tabs, 1.0, SIXPI, 1.0)
            assert K.pp_shapes()[1] == k
            assert _rel_rms((got - img.vp).astype(np.float64), dv_want) < 1e-6, table[k]
            assert abs(f2 - f2_want) <= 1e-5 * f2_want, table[k]
            np.testing.assert_allclose(vmax, vmax_want, rtol=1e-5)
    finally:
        K.pp_set_shape(-1)


def test_autotuner_times_every_shape_once_and_keeps_the_fastest(gpu, clumpy):
    from cube2_b200 import kick as K
    img, tabs = clumpy
    fk = K.FineKick(img.layout, pm3_mode=K.CUBE_PM3_PERIODIC)
    K.pp_set_shape(-1)  # forget earlier picks
    want, _, _, _, _ = fk.c_pp_force_kernel(img, *tabs, 1.0, SIXPI, 1.0)
    table, cur = K.pp_shapes()
    ms = np.array([t["ms"] for t in table])
    assert np.all(ms > 0)
    assert cur == int(np.argmin(ms))
    # the same key: no new timing, same shape, same kick
    got, _, _, _, _ = fk.c_pp_force_kernel(img, *tabs, 1.0, SIXPI, 1.0)
    table2, cur2 = K.pp_shapes()
    assert cur2 == cur
    assert [t["ms"] for t in table2] == [t["ms"] for t in table]
    np.testing.assert_array_equal(got, want)

