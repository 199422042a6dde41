"""Learned PP shell: the CPU oracle's gradients against finite differences (no GPU)."""
import numpy as np

from oracle import mlp_oracle as M


def test_oracle_backward_matches_finite_differences(monkeypatch):
    # without the BF16 rounding the oracle's loss is smooth, so central differences apply
    monkeypatch.setattr(M, "bf16", lambda a: np.asarray(a, dtype=np.float64))
    rng = np.random.default_rng(3)
    p = {k: v.astype(np.float64) for k, v in M.init_params(5).items()}
    X = rng.standard_normal((12, M.K_PAD))
    X[:, M.K_IN:] = 0.0
    T = rng.standard_normal((12, 3))
    y, cache = M.forward(p, X)
    _, g = M.backward(p, cache, y, T)
    eps = 1e-6
    for name in ("W1", "b1", "W2", "b3", "W4", "b4"):
        for idx in [tuple(rng.integers(0, s) for s in p[name].shape) for _ in range(4)]:
            if name == "W1" and idx[1] >= M.K_IN:
                continue
            old = p[name][idx]
            p[name][idx] = old + eps
            lp = float(np.mean((M.forward(p, X)[0] - T) ** 2))
            p[name][idx] = old - eps
            lm = float(np.mean((M.forward(p, X)[0] - T) ** 2))
            p[name][idx] = old
            num = (lp - lm) / (2 * eps)
            assert abs(num - g[name][idx]) <= 1e-6 + 1e-4 * abs(num), (name, idx, num, g[name][idx])


def test_oracle_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5e-3, 3.0e38])
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie goes to the even mantissa
    assert r[2] == 1.0 + 2 ** -7
    assert abs(r[3] - -2.5e-3) <= 2.5e-3 * 2 ** -8
    assert np.isfinite(r[4])


def test_package_parameter_layout_matches_oracle():
    from cube2_b200 import learned as Ln
    flat = Ln.init_params(7)
    assert flat.size == Ln.N_PARAMS == 43779
    p = Ln.unflatten(flat)
    assert p["W1"].shape == (128, 80) and np.all(p["W1"][:, 67:] == 0)
    assert p["W4"].shape == (3, 128) and p["b4"].shape == (3,)
    np.testing.assert_array_equal(Ln.flatten(p), flat)
