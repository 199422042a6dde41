"""Learned PP shell on the GPU against its CPU oracle (oracle/mlp_oracle.py).

Features, the BF16 tensor-core forward, the gradients of one training step, the Adam
update and the fused inference + kick are checked against the oracle on the same inputs;
then a short training run shows what the trained network gains over the cutoff-1 kick
without it on held-out particles.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel_rms(a, b):
    return float(np.sqrt(np.sum((np.asarray(a, np.float64) - b) ** 2) / np.sum(np.asarray(b, np.float64) ** 2)))


def _zeld():
    import torch
    from cube2_b200 import learned as Ln
    from cube2_b200 import workloads as W
    img = W.make("zeldovich64")
    dev = torch.device("cuda:0")
    rho, idx, xp, vp = Ln.device_image(img, dev)
    return img, rho, idx, xp, vp


def test_mlp_features_match_oracle(gpu):
    from cube2_b200 import learned as Ln
    from cube2_b200 import workloads as W
    from oracle import mlp_oracle as M
    img, rho, idx, xp, _ = _zeld()
    X = Ln.features(img.layout, rho, idx, xp, img.n_used).float().cpu().numpy()
    pos = W.physical_positions(img)
    act = np.nonzero(img.active)[0]
    dens = M.cic_density(pos, img.layout.ng)
    ref = M.features(pos[img.pid[act]], dens)
    assert np.all(X[~img.active] == 0)
    np.testing.assert_allclose(X[act], M.bf16(ref), rtol=1e-2, atol=1e-3)


def test_mlp_forward_gradients_and_adam_match_oracle(gpu):
    import torch
    from cube2_b200 import learned as Ln
    from oracle import mlp_oracle as M
    img, rho, idx, xp, _ = _zeld()
    dev = rho.device
    X = Ln.features(img.layout, rho, idx, xp, img.n_used)
    act = np.nonzero(img.active)[0]
    rng = np.random.default_rng(11)
    rows = np.sort(rng.choice(act, 256, replace=False)).astype(np.int32)
    Xh = X.float().cpu().numpy()
    flat = Ln.init_params(2)
    p = {k: v.copy() for k, v in Ln.unflatten(flat).items()}
    for k in ("b1", "b2", "b3", "b4"):
        p[k] = (0.1 * rng.standard_normal(p[k].shape)).astype(np.float32)
    flat = Ln.flatten(p)
    net = Ln.ShellNet(flat, batch_cap=256)
    # forward
    Y = torch.zeros((256, 3), device=dev)
    Xr = X[torch.from_numpy(rows.astype(np.int64)).to(dev)]
    net.forward(Xr, 256, Y)
    torch.cuda.synchronize()
    y_ref, cache = M.forward(p, Xh[rows])
    assert _rel_rms(Y.cpu().numpy(), y_ref) < 1e-2
    # one Adam step: its gradients, then the update
    T = rng.standard_normal((img.n_used, 3)).astype(np.float32)
    dT = torch.from_numpy(T).to(dev)
    loss = torch.zeros(1, device=dev)
    net.train_step(X, dT, torch.from_numpy(rows).to(dev), 256, 1e-3, loss)
    torch.cuda.synchronize()
    lref, g = M.backward(p, cache, y_ref, T[rows])
    assert abs(float(loss.item()) - lref) <= 1e-2 * lref
    got = Ln.unflatten(net.grads())
    for k in g:
        assert _rel_rms(got[k], g[k]) < 3e-2, k
    m = {k: np.zeros_like(v, np.float64) for k, v in p.items()}
    v = {k: np.zeros_like(w, np.float64) for k, w in p.items()}
    pref = {k: w.astype(np.float64) for k, w in p.items()}
    M.adam(pref, {k: got[k].astype(np.float64) for k in got}, m, v, 1, 1e-3)
    after = Ln.unflatten(net.params())
    for k in pref:
        np.testing.assert_allclose(after[k], pref[k], rtol=1e-5, atol=1e-7)
    net.close()


def test_mlp_kick_equals_forward(gpu):
    """The fused inference + kick adds kick * scale * forward(features) to the interior copies."""
    import torch
    from cube2_b200 import learned as Ln
    img, rho, idx, xp, vp = _zeld()
    dev = rho.device
    net = Ln.ShellNet(Ln.init_params(4), batch_cap=4096)
    X = Ln.features(img.layout, rho, idx, xp, img.n_used)
    Y = torch.zeros((img.n_used, 3), device=dev)
    net.forward(X, img.n_used, Y)
    vp0 = vp.clone()
    net.kick(rho, idx, xp, img.n_used, vp, 0.5, 6 * np.pi, 1.0)
    torch.cuda.synchronize()
    dv = (vp - vp0).cpu().numpy().reshape(-1, 3)
    want = 0.5 * Ln.kick_coef(6 * np.pi, 1.0) * Y.cpu().numpy()
    assert np.all(dv[~img.active] == 0)
    assert _rel_rms(dv[img.active], want[img.active]) < 2e-3
    net.close()


def test_trained_shell_gains_over_cutoff_one(gpu):
    """Train on two clustered boxes, measure on a third: the network must explain a clear part of
    the force the cutoff-1 split misses (the method without it explains none)."""
    import torch
    from cube2_b200 import ic
    from cube2_b200 import learned as Ln
    from cube2_b200.layout import RATIO_SF, Layout, build_image, ixyz3_table
    L = Layout(ng=64, nnt=1, nns=2, ratio_cs=4, ngb=4, app=0.1)
    tabs = (np.arange(1, L.ns3 + 1, dtype=np.int32), np.full(L.ns3, 2, np.int32), ixyz3_table(L), None, RATIO_SF)
    imgs = [build_image(*ic.lognormal_poisson(64, s, seed)[:2], L) for s, seed in ((1.0, 4002), (1.5, 4003),
                                                                                   (1.5, 4013))]
    dev = torch.device("cuda:0")
    X, T, scale = Ln.training_set(imgs, [tabs] * 3, dev)
    ntest = int(np.sum(imgs[2].active))
    ntrain = X.shape[0] - ntest
    Xs, mu, sd = Ln.standardize(X, ntrain)
    net = Ln.ShellNet(batch_cap=4096, seed=1)
    Ln.train(net, Xs, T, steps=3000, batch=4096, lr=1e-3, holdout=ntrain)
    test_rows = torch.arange(ntrain, X.shape[0], device=dev)
    u = Ln.unexplained(net, Xs, T, test_rows)
    assert u < 0.9, u  # measured 0.86: the network recovers ~14% of the missing force variance
    # folded into the first layer, the network gives the same outputs on raw inputs
    raw = Ln.ShellNet(Ln.fold(net.params(), mu, sd), batch_cap=4096)
    u_raw = Ln.unexplained(raw, X, T, test_rows)
    assert abs(u_raw - u) < 0.02, (u, u_raw)
    net.close()
    raw.close()


def test_tensor_memory_kernel_matches_mma_sync_kernel(gpu, monkeypatch):
    """The inference kernel on tcgen05 (accumulators in tensor memory) against the mma.sync one,
    on the same features and weights: both round the activations to BF16, so they agree to the
    accumulation order."""
    import torch
    from cube2_b200 import learned as Ln
    img, rho, idx, xp, vp = _zeld()
    rng = np.random.default_rng(8)
    p = Ln.unflatten(Ln.init_params(9))
    for k in ("b1", "b2", "b3", "b4"):
        p[k] = (0.1 * rng.standard_normal(p[k].shape)).astype(np.float32)
    net = Ln.ShellNet(Ln.flatten(p), batch_cap=256)
    out = []
    for mma_sync in (False, True):
        if mma_sync:
            monkeypatch.setenv("CUBE_MLP_MMA_SYNC", "1")
        v = vp.clone()
        net.kick(rho, idx, xp, img.n_used, v, 1.0, 6 * np.pi, 1.0)
        torch.cuda.synchronize()
        out.append((v - vp).cpu().numpy().reshape(-1, 3))
    monkeypatch.delenv("CUBE_MLP_MMA_SYNC")
    assert np.all(out[0][~img.active] == 0)
    assert _rel_rms(out[0][img.active], out[1][img.active]) < 2e-3
    net.close()
