"""Learned PP shell: the network handle, its training on the GPU and the learned kick.

The shell lets the PP cutoff drop from 2 to 1 fine cells: the kick becomes the plain
machinery run with PM3 softened at 1 fine cell (apm3f = 2 mesh cells) and PP within
1 fine cell, plus a small MLP (cube_mlp_*, csrc/mlp.cu) that predicts, per particle, the
force the cutoff-1 split misses against the cutoff-2 split.  The network is trained on
forces the method itself produces: for a training image, the target of a particle is
(cutoff-2 kick - cutoff-1 kick) / kick coefficient, in units of the rms target.

Everything runs through the library's C ABI on device arrays (torch tensors as device
memory only): feature rows (cube_mlp_features), Adam steps on random batches
(cube_mlp_train_step), the fused inference + kick (cube_mlp_kick).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from .kick import CUBE_PM3_PERIODIC, FineKick, _check, _p, lib
from .layout import Image, Layout, apm3_table

N_PARAMS = 43779
K_IN, K_PAD, WIDTH, N_OUT = 67, 80, 128, 3
_SHAPES = [("W1", (WIDTH, K_PAD)), ("b1", (WIDTH,)), ("W2", (WIDTH, WIDTH)), ("b2", (WIDTH,)),
           ("W3", (WIDTH, WIDTH)), ("b3", (WIDTH,)), ("W4", (N_OUT, WIDTH)), ("b4", (N_OUT,))]


def unflatten(flat: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shp in _SHAPES:
        n = int(np.prod(shp))
        out[name] = flat[o:o + n].reshape(shp)
        o += n
    return out


def flatten(p: dict) -> np.ndarray:
    return np.concatenate([np.asarray(p[name], np.float32).reshape(-1) for name, _ in _SHAPES]).astype(np.float32)


def init_params(seed: int = 0) -> np.ndarray:
    """He initialisation (W1 reads the 67 real inputs of the 80 padded ones), zero biases."""
    rng = np.random.default_rng(seed)
    p = {}
    for name, shp in _SHAPES:
        if name.startswith("W"):
            fan = K_IN if name == "W1" else shp[1]
            W = rng.standard_normal(shp) * np.sqrt(2.0 / fan)
            if name == "W1":
                W[:, K_IN:] = 0.0
            p[name] = W.astype(np.float32)
        else:
            p[name] = np.zeros(shp, np.float32)
    return flatten(p)


def _dp(x):
    return ctypes.c_void_p(x if isinstance(x, int) else x.data_ptr())


def _sp(stream):
    return None if stream is None else ctypes.c_void_p(stream if isinstance(stream, int) else stream.cuda_stream)


class ShellNet:
    """The network on the device (cube_mlp_create); training batches up to `batch_cap` rows."""

    def __init__(self, params: np.ndarray | None = None, batch_cap: int = 8192, seed: int = 0):
        flat = init_params(seed) if params is None else np.ascontiguousarray(params, np.float32)
        if flat.size != N_PARAMS:
            raise ValueError("wrong parameter count")
        self.batch_cap = batch_cap
        h = ctypes.c_void_p()
        _check(lib().cube_mlp_create(_p(flat), ctypes.c_int32(batch_cap), ctypes.byref(h)), "cube_mlp_create")
        self.h = h

    def params(self) -> np.ndarray:
        out = np.zeros(N_PARAMS, np.float32)
        _check(lib().cube_mlp_get_params(self.h, _p(out), None), "cube_mlp_get_params")
        return out

    def grads(self) -> np.ndarray:
        out = np.zeros(N_PARAMS, np.float32)
        _check(lib().cube_mlp_get_params(self.h, None, _p(out)), "cube_mlp_get_params")
        return out

    def train_step(self, d_X, d_T, d_rows, batch: int, lr: float, d_loss, stream=None):
        _check(lib().cube_mlp_train_step(self.h, _dp(d_X), _dp(d_T), _dp(d_rows), ctypes.c_int32(batch),
                                         ctypes.c_float(lr), _dp(d_loss), _sp(stream)), "cube_mlp_train_step")

    def forward(self, d_X, rows: int, d_Y, stream=None):
        _check(lib().cube_mlp_forward(self.h, _dp(d_X), ctypes.c_int64(rows), _dp(d_Y), _sp(stream)),
               "cube_mlp_forward")

    def kick(self, d_rhoc, d_idx, d_xp, n_used: int, d_vp, scale: float, a_mid: float, dt: float, stream=None):
        _check(lib().cube_mlp_kick(self.h, _dp(d_rhoc), _dp(d_idx), _dp(d_xp), ctypes.c_int64(n_used), _dp(d_vp),
                                   ctypes.c_float(scale), ctypes.c_float(a_mid), ctypes.c_float(dt), _sp(stream)),
               "cube_mlp_kick")

    def close(self):
        if self.h:
            lib().cube_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def features(layout: Layout, d_rhoc, d_idx, d_xp, n_used: int, stream=None):
    """BF16 input rows [n_used][80] of the configured image (torch tensor; zeros for buffer copies)."""
    import torch
    X = torch.zeros((max(n_used, 1), K_PAD), dtype=torch.bfloat16, device=d_xp.device)
    FineKick(layout, pm3_mode=CUBE_PM3_PERIODIC)
    _check(lib().cube_mlp_features(_dp(d_rhoc), _dp(d_idx), _dp(d_xp), ctypes.c_int64(n_used), _dp(X),
                                   _sp(stream)), "cube_mlp_features")
    return X


def fallback(d_rhoc, d_idx, n_used: int, d_vp0, d_vp_learned, d_vp_full, bound: float, samples: int = 4,
             d_vp_out=None, stream=None) -> dict:
    """Per-cell check of the learned kick against the full-cutoff kick and fallback of the cells
    over the bound (cube_learned_fallback); d_vp_out defaults to d_vp_learned (in place)."""
    out = np.zeros(5, np.float64)
    dst = d_vp_learned if d_vp_out is None else d_vp_out
    _check(lib().cube_learned_fallback(_dp(d_rhoc), _dp(d_idx), ctypes.c_int64(int(n_used)), _dp(d_vp0),
                                       _dp(d_vp_learned), _dp(d_vp_full), ctypes.c_float(bound),
                                       ctypes.c_int32(samples), _dp(dst), _p(out), _sp(stream)),
           "cube_learned_fallback")
    return dict(cells_checked=int(out[0]), cells_over=int(out[1]), particles_fallen_back=int(out[2]),
                sampled_rms_vs_full=float(out[3]), samples=int(out[4]))


def kick_coef(a_mid: float, dt: float) -> float:
    return float(np.float32(np.float32(a_mid) * np.float32(dt) / np.float32(6.0))) / np.pi


@dataclass
class Split:
    """PP cutoff (fine cells) and PM3 softening (mesh cells on the ratio_sf = 2 mesh) of a kick."""
    apm3f: float

    @property
    def cutoff(self) -> float:
        return self.apm3f / 2.0


PLAIN, SHORT = Split(4.0), Split(2.0)


def device_image(img: Image, device):
    import torch

    def up(a):
        return torch.from_numpy(np.ascontiguousarray(a).reshape(-1).copy()).to(device)
    return up(img.rhoc), up(img.idx_b_r), up(img.xp), up(img.vp)


def split_forces(img: Image, tables, split: Split, device, stream=None) -> np.ndarray:
    """Per stored copy, the force of one kick with this split (dv / kick coefficient; 0 for buffers)."""
    import torch
    isort, ires, ix, _, rs = tables
    fk = FineKick(img.layout, pm3_mode=CUBE_PM3_PERIODIC, apm3f=split.apm3f)
    rho, idx, xp, vp = device_image(img, device)
    vp0 = vp.clone()
    out = torch.zeros(8, device=device)
    fk.kick_fine_device(rho, idx, xp, img.n_used, vp, out, isort, ires, ix, apm3_table(split.apm3f), rs, 1.0,
                        6 * np.pi, 1.0, stream=stream)
    torch.cuda.synchronize()
    return ((vp - vp0).cpu().numpy().reshape(-1, 3).astype(np.float64) / kick_coef(6 * np.pi, 1.0))


def training_set(images, tables_list, device, stream=None):
    """Inputs, targets (in units of the target rms) and the rows of interior copies of several
    images, stacked; returns (X bf16 [rows][80], T f32 [rows][3], scale)."""
    import torch
    Xs, Ts = [], []
    for img, tabs in zip(images, tables_list):
        f2 = split_forces(img, tabs, PLAIN, device, stream)
        f1 = split_forces(img, tabs, SHORT, device, stream)
        act = np.nonzero(img.active)[0]
        rho, idx, xp, _ = device_image(img, device)
        X = features(img.layout, rho, idx, xp, img.n_used, stream)
        torch.cuda.synchronize()
        Xs.append(X[torch.from_numpy(act).to(device)])
        Ts.append((f2 - f1)[act])
    T = np.concatenate(Ts)
    scale = float(np.sqrt(np.mean(np.sum(T * T, axis=1)) / 3.0))
    return torch.cat(Xs), torch.from_numpy((T / scale).astype(np.float32)).to(device), scale


def standardize(X, rows: int):
    """Inputs scaled to zero mean and unit variance over the first `rows` rows (the padding
    columns stay 0); returns (Xs, mean, std).  Training runs on Xs, and fold() moves the
    scaling into the first layer for the kick, which reads raw inputs."""
    import torch
    Xf = X[:rows].float()
    mu = Xf.mean(0)
    sd = Xf.std(0)
    mu[K_IN:] = 0.0
    sd[K_IN:] = 1.0
    sd = torch.where(sd > 1e-6, sd, torch.ones_like(sd))
    return ((X.float() - mu) / sd).to(torch.bfloat16), mu.cpu().numpy(), sd.cpu().numpy()


def fold(flat: np.ndarray, mu: np.ndarray, sd: np.ndarray) -> np.ndarray:
    """Parameters of a network trained on standardized inputs, rewritten for raw inputs:
    W1 x' + b1 with x' = (x - mu) / sd equals (W1 / sd) x + (b1 - (W1 / sd) mu)."""
    p = unflatten(flat.astype(np.float64))
    W1 = p["W1"] / sd[None, :]
    p["b1"] = p["b1"] - W1 @ mu
    p["W1"] = W1
    return flatten(p)


def train(net: ShellNet, X, T, steps: int, batch: int = 4096, lr: float = 1e-3, seed: int = 0, holdout=None,
          log_every: int = 0, stream=None):
    """Adam on random batches of rows (cosine learning-rate decay); returns the loss history."""
    import torch
    dev = X.device
    g = torch.Generator(device="cpu").manual_seed(seed)
    n = X.shape[0] if holdout is None else holdout
    loss = torch.zeros(1, device=dev)
    hist = []
    since = 0
    for k in range(steps):
        rows = torch.randint(0, n, (batch,), generator=g, dtype=torch.int32).to(dev)
        lr_k = 0.5 * lr * (1.0 + np.cos(np.pi * k / max(steps, 1)))
        net.train_step(X, T, rows, batch, lr_k, loss, stream)  # adds this batch's mean loss
        since += 1
        if log_every and ((k + 1) % log_every == 0 or k == steps - 1):
            torch.cuda.synchronize()
            hist.append((k + 1, float(loss.item()) / since))  # mean batch loss since the last entry
            loss.zero_()
            since = 0
    torch.cuda.synchronize()
    return hist


def unexplained(net: ShellNet, X, T, rows) -> float:
    """Fraction of the target variance the network leaves unexplained on `rows`."""
    import torch
    Xr, Tr = X[rows], T[rows]
    Y = torch.zeros((Xr.shape[0], 3), dtype=torch.float32, device=X.device)
    net.forward(Xr, Xr.shape[0], Y)
    torch.cuda.synchronize()
    r = (Tr - Y).double()
    return float((r * r).sum() / (Tr.double() ** 2).sum())


def train_shell_on(images, device, steps: int = 6000, batch: int = 8192, seed: int = 1, fields: str = ""):
    """A shell trained on the method's own forces on `images` (host Images in the periodic
    layout): targets from the cutoff-2 and cutoff-1 kicks of each image, Adam on standardized
    inputs, folded for raw inputs.  Returns (ShellNet, target scale, info)."""
    import time

    from .layout import RATIO_SF, ixyz3_table
    t0 = time.perf_counter()
    tabs = [(np.arange(1, im.layout.ns3 + 1, dtype=np.int32), np.full(im.layout.ns3, 2, np.int32),
             ixyz3_table(im.layout), None, RATIO_SF) for im in images]
    X, T, scale = training_set(images, tabs, device)
    Xs, mu, sd = standardize(X, X.shape[0])
    net = ShellNet(batch_cap=batch, seed=seed)
    hist = train(net, Xs, T, steps=steps, batch=batch, lr=1e-3, log_every=1000)
    shell = ShellNet(fold(net.params(), mu, sd), batch_cap=16)
    net.close()
    info = {"samples": int(X.shape[0]), "steps": steps, "batch": batch, "seconds": time.perf_counter() - t0,
            "loss": hist, "fields": fields}
    del X, Xs, T
    return shell, scale, info


def train_shell(device, steps: int = 6000, batch: int = 8192, seed: int = 1):
    """The shell of the single-kick benchmark: trained on three lognormal Poisson boxes of 96^3
    fine cells (sigma 0.5, 1.0, 1.5; seeds 4001..4003, about 2.6M samples)."""
    from . import ic
    from .layout import build_image
    Lt = Layout(ng=96, nnt=1, nns=2, ratio_cs=4, ngb=4, app=0.1)
    boxes = [build_image(*ic.lognormal_poisson(96, sg, sd)[:2], Lt) for sg, sd in ((0.5, 4001), (1.0, 4002),
                                                                                   (1.5, 4003))]
    return train_shell_on(boxes, device, steps, batch, seed,
                          fields="lognormal Poisson 96^3, sigma 0.5 / 1.0 / 1.5 (seeds 4001..4003)")
