"""CPU oracle of the learned PP shell (test infrastructure: used by tests/ only).

The learned shell has no counterpart in the reference; its definition lives in
cube2_b200/csrc/mlp.cu and this module restates it in numpy (float64 arithmetic
on BF16-rounded operands, the rounding of the device kernels), so that the device
forward, backward and Adam kernels can be checked value by value.

* Features of a particle at fine-cell position x (periodic box of ng cells): the
  CIC density of all particles on the fine grid (cell centres at i + 0.5), read on
  the 4^3 cells i0-1 .. i0+2 around i0 = floor(x - 0.5) (x fastest), as log(1 + rho),
  then the 3 offsets f = x - 0.5 - i0; 67 inputs, zero-padded to 80.
* Network: h1 = gelu(W1 x + b1), h2 = gelu(W2 h1 + b2), h3 = gelu(W3 h2 + b3),
  y = W4 h3 + b4 with widths 128, 128, 128, 3; gelu(z) = z/2 (1 + tanh(c (z + 0.044715 z^3))),
  c = sqrt(2/pi).  Every GEMM operand (x, W, h) is rounded to BF16; accumulation and
  biases are FP32 or wider.
* Loss: mean over samples and components of (y - t)^2; Adam with bias correction.
"""
from __future__ import annotations

import numpy as np

K_IN = 67
K_PAD = 80
WIDTH = 128
N_OUT = 3
GELU_C = np.sqrt(2.0 / np.pi)


def bf16(a: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def cic_density(pos: np.ndarray, ng: int) -> np.ndarray:
    """CIC density [z][y][x] of unit-mass particles on the periodic fine grid."""
    rho = np.zeros((ng, ng, ng))
    xs = pos - 0.5
    i0 = np.floor(xs).astype(np.int64)
    f = xs - i0
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                w = (f[:, 0] if dx else 1 - f[:, 0]) * (f[:, 1] if dy else 1 - f[:, 1]) * \
                    (f[:, 2] if dz else 1 - f[:, 2])
                np.add.at(rho, ((i0[:, 2] + dz) % ng, (i0[:, 1] + dy) % ng, (i0[:, 0] + dx) % ng), w)
    return rho


def features(pos: np.ndarray, rho: np.ndarray) -> np.ndarray:
    """[n][K_PAD] inputs of particles at `pos` on the density `rho`."""
    ng = rho.shape[0]
    xs = pos - 0.5
    i0 = np.floor(xs).astype(np.int64)
    f = xs - i0
    X = np.zeros((pos.shape[0], K_PAD))
    k = 0
    for dz in range(-1, 3):
        for dy in range(-1, 3):
            for dx in range(-1, 3):
                X[:, k] = np.log1p(rho[(i0[:, 2] + dz) % ng, (i0[:, 1] + dy) % ng, (i0[:, 0] + dx) % ng])
                k += 1
    X[:, 64:67] = f
    return X


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(GELU_C * (z + 0.044715 * z ** 3)))


def gelu_grad(z):
    t = np.tanh(GELU_C * (z + 0.044715 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GELU_C * (1.0 + 3 * 0.044715 * z * z)


def init_params(seed: int = 0) -> dict:
    """He-style initialisation in FP32 (W1 reads the K_PAD padded inputs)."""
    rng = np.random.default_rng(seed)
    p = {}
    dims = [(WIDTH, K_PAD), (WIDTH, WIDTH), (WIDTH, WIDTH), (N_OUT, WIDTH)]
    for i, (o, k) in enumerate(dims, 1):
        fan = K_IN if i == 1 else k
        W = rng.standard_normal((o, k)) * np.sqrt(2.0 / fan)
        if i == 1:
            W[:, K_IN:] = 0.0
        p[f"W{i}"] = W.astype(np.float32)
        p[f"b{i}"] = np.zeros(o, np.float32)
    return p


def forward(p: dict, X: np.ndarray):
    """Returns y and the cache (pre-activations and BF16 layer inputs) for backward."""
    a = bf16(X)
    cache = {"a0": a}
    for i in (1, 2, 3):
        z = a @ bf16(p[f"W{i}"]).T + p[f"b{i}"].astype(np.float64)
        cache[f"z{i}"] = z
        a = bf16(gelu(z))
        cache[f"a{i}"] = a
    y = a @ bf16(p["W4"]).T + p["b4"].astype(np.float64)
    return y, cache


def backward(p: dict, cache: dict, y: np.ndarray, t: np.ndarray) -> tuple[float, dict]:
    """MSE loss and its gradients; dL/dy = 2 (y - t) / (n * 3)."""
    n = y.shape[0]
    loss = float(np.mean((y - t) ** 2))
    dy = 2.0 * (y - t) / (n * N_OUT)
    g = {"W4": bf16(dy).T @ cache["a3"], "b4": dy.sum(0)}
    da = bf16(dy) @ bf16(p["W4"])
    for i in (3, 2, 1):
        dz = da * gelu_grad(cache[f"z{i}"])
        g[f"W{i}"] = bf16(dz).T @ cache[f"a{i - 1}"]
        g[f"b{i}"] = dz.sum(0)
        if i > 1:
            da = bf16(dz) @ bf16(p[f"W{i}"])
    return loss, g


def adam(p: dict, g: dict, m: dict, v: dict, step: int, lr: float, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step in place on FP32 parameters (step counts from 1)."""
    for k in p:
        m[k] = b1 * m[k] + (1 - b1) * g[k]
        v[k] = b2 * v[k] + (1 - b2) * g[k] * g[k]
        mh = m[k] / (1 - b1 ** step)
        vh = v[k] / (1 - b2 ** step)
        p[k] = (p[k] - lr * mh / (np.sqrt(vh) + eps)).astype(np.float32)
