"""ORACLE -- test infrastructure only.

CPU restatement of the CIC power spectrum: the deposit of utilities/cicpower.f90:55-70
(position * nw / nc - 0.5 on a cell-centred periodic grid, lower weight idx1 - x, upper
weight x - idx1 + 1), delta = rho nw^3 / N - 1, delta_k = FFT / nw^3, and the linear-k
binning of utilities/powerspectrum.f90:52-94 (half spectrum without the conjugate
duplicates of the i = 0 and i = nyquist planes, bin nint(|k|), CIC window sinc^4).
"""
import numpy as np


def cic_grid(pos_coarse: np.ndarray, nc: int, nw: int) -> np.ndarray:
    """Deposit of unit masses at coarse-cell positions in [0, nc) on a [z][y][x] nw^3 grid."""
    x = pos_coarse.astype(np.float64) * (nw / nc) - 0.5
    i0 = np.floor(x).astype(np.int64)
    w1 = x - i0
    grid = np.zeros(nw ** 3, np.float64)
    for k in range(8):
        d = np.array([k & 1, (k >> 1) & 1, k >> 2])
        idx = np.mod(i0 + d, nw)
        w = np.prod(np.where(d == 1, w1, 1.0 - w1), axis=1)
        np.add.at(grid, (idx[:, 2] * nw + idx[:, 1]) * nw + idx[:, 0], w)
    return grid.reshape(nw, nw, nw)


def power_spectrum(pos_coarse: np.ndarray, nc: int, nw: int, nbin: int = 0) -> dict:
    nb = nbin if nbin > 0 else int(round((nw // 2) * np.sqrt(3.0)))
    rho = cic_grid(pos_coarse, nc, nw)
    delta = rho * (nw ** 3 / pos_coarse.shape[0]) - 1.0
    ck = np.fft.rfftn(delta) / nw ** 3
    nyq = nw // 2
    k = np.arange(nw)
    kk = np.mod(k + nyq, nw) - nyq
    kz, ky, kx = np.meshgrid(kk, kk, kk[:nyq + 1], indexing="ij")
    i = np.broadcast_to(np.arange(nyq + 1)[None, None, :], kx.shape)
    j = np.broadcast_to(np.arange(nw)[None, :, None], kx.shape)
    kq = np.broadcast_to(np.arange(nw)[:, None, None], kx.shape)
    keep = ~((i == 0) & (j == 0) & (kq == 0))
    keep &= ~(((i == 0) | (i == nyq)) & (j > nyq))
    keep &= ~(((i == 0) | (i == nyq)) & ((j == 0) | (j == nyq)) & (kq > nyq))
    kr = np.sqrt(kx.astype(np.float64) ** 2 + ky ** 2 + kz ** 2)
    b = np.rint(kr).astype(np.int64)
    keep &= b <= nb

    def sinc(q):
        a = np.pi * q / nw
        return np.where(q == 0, 1.0, np.sin(np.where(q == 0, 1.0, a)) / np.where(q == 0, 1.0, a))
    s = sinc(kx) * sinc(ky) * sinc(kz)
    pk = np.abs(ck) ** 2 / s ** 4
    out = np.zeros((4, nb + 1))
    for row, val in enumerate((np.ones_like(kr), kr, pk, pk * 4 * np.pi * kr ** 3)):
        out[row] = np.bincount(b[keep], weights=val[keep], minlength=nb + 1)
    modes = out[0]
    with np.errstate(invalid="ignore", divide="ignore"):
        return {"modes": modes, "k": out[1] / modes, "pk": out[2] / modes, "delta2": out[3] / modes}
