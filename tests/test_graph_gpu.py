"""The device kick captured as one CUDA graph (cube_kick_graph_*).

A replay must give the kick of cube_kick_fine_device on the same arrays (within float
atomics' reordering), creation must leave vp untouched, and the subtile geometry, whose
mesh batches synchronise the host, is refused.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIXPI = float(np.float32(6 * np.pi))
TOL = 1e-6


def _rel_rms(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def _device(img):
    import torch
    dev = torch.device("cuda:0")

    def up(a):
        return torch.from_numpy(np.ascontiguousarray(a).reshape(-1).copy()).to(dev)
    return up(img.rhoc), up(img.idx_b_r), up(img.xp), up(img.vp), torch.zeros(8, device=dev)


@pytest.mark.parametrize("name", ["zeldovich64", "batch8"])
def test_graph_replays_equal_direct_kicks(gpu, name):
    import torch
    from cube2_b200 import workloads as W
    from cube2_b200.kick import CUBE_PM3_PERIODIC, CUBE_PM3_TILE_PERIODIC, FineKick
    img = W.make(name)
    tabs = W.tables(name)
    mode = CUBE_PM3_TILE_PERIODIC if W.WORKLOADS[name]["kind"] == "batch" else CUBE_PM3_PERIODIC
    fk = FineKick(img.layout, pm3_mode=mode, apm3f=4.0)
    s = torch.cuda.Stream()
    # two direct kicks
    rho, idx, xp, vp, out = _device(img)
    for _ in range(2):
        fk.kick_fine_device(rho, idx, xp, img.n_used, vp, out, *tabs, 1.0, SIXPI, 1.0, stream=s)
    torch.cuda.synchronize()
    want, want_out = vp.cpu().numpy().reshape(-1, 3), out.cpu().numpy()
    # a graph of the same kick, replayed twice
    rho2, idx2, xp2, vp2, out2 = _device(img)
    graph = fk.kick_graph(rho2, idx2, xp2, img.n_used, vp2, out2, *tabs, 1.0, SIXPI, 1.0)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(vp2.cpu().numpy().reshape(-1, 3), img.vp)  # creation kicks a scratch copy
    graph.launch(s)
    graph.launch(s)
    torch.cuda.synchronize()
    got = vp2.cpu().numpy().reshape(-1, 3)
    assert _rel_rms((got - img.vp).astype(np.float64), (want - img.vp).astype(np.float64)) < TOL
    o = out2.cpu().numpy()
    assert o[5:6].view(np.int32)[0] == 0
    np.testing.assert_allclose(o[:5], want_out[:5], rtol=1e-5)
    graph.close()


def test_graph_refuses_subtile_geometry(gpu):
    from cube2_b200 import workloads as W
    from cube2_b200.kick import CUBE_PM3_SUBTILE, CubeError, FineKick
    img = W.make("zeldovich64")
    fk = FineKick(img.layout, pm3_mode=CUBE_PM3_SUBTILE, apm3f=4.0)
    rho, idx, xp, vp, out = _device(img)
    with pytest.raises(CubeError):
        fk.kick_graph(rho, idx, xp, img.n_used, vp, out, *W.tables("zeldovich64"), 1.0, SIXPI, 1.0)
