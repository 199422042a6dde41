"""Seeded synthetic particle sets for the fine-scale kick workloads.

All generators use ``numpy.random.Generator(PCG64(seed))`` and return
positions in fine-cell units in [0, L) and float32 velocities.  They stand
in for CUBE2's initial-condition program (utilities/ic.f90), whose transfer
functions need CAMB tables; only the statistics named by each workload are
reproduced (power-law Gaussian fields, Zel'dovich displacement, lognormal
Poisson sampling).
"""
from __future__ import annotations

import numpy as np


def _kgrid(n: int):
    k1 = np.fft.fftfreq(n) * n
    kr = np.fft.rfftfreq(n) * n
    return k1[:, None, None], k1[None, :, None], kr[None, None, :]


def gaussian_field(n: int, slope: float, rng: np.random.Generator) -> np.ndarray:
    """Real Gaussian random field on n^3 with P(k) proportional to k^slope (k != 0), unit variance."""
    white = rng.standard_normal((n, n, n))
    wk = np.fft.rfftn(white)
    kz, ky, kx = _kgrid(n)
    k2 = kx * kx + ky * ky + kz * kz
    amp = np.zeros_like(k2)
    nz = k2 > 0
    amp[nz] = k2[nz] ** (slope / 4.0)
    f = np.fft.irfftn(wk * amp, s=(n, n, n), axes=(0, 1, 2))
    f -= f.mean()
    return f / f.std()


def zeldovich_lattice(n: int, rms_disp: float, seed: int, slope: float = -2.0):
    """Lattice at cell centres displaced by the Zel'dovich field of a P ~ k^slope Gaussian delta.

    Psi(k) = i k delta(k) / k^2, scaled so that rms |Psi| = rms_disp cells.
    Returns (pos float64[n^3,3] in [0,n), vel float32[n^3,3] = Psi, delta field).
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    delta = gaussian_field(n, slope, rng)
    dk = np.fft.rfftn(delta)
    kz, ky, kx = _kgrid(n)
    k2 = kx * kx + ky * ky + kz * kz
    k2[0, 0, 0] = 1.0
    psi = []
    for kc in (kx, ky, kz):
        comp = np.fft.irfftn(1j * kc * dk / k2 * (n / (2 * np.pi)), s=(n, n, n), axes=(0, 1, 2))
        psi.append(comp)
    psi = np.stack(psi, axis=-1)  # [z,y,x,3] components (x,y,z)
    rms = np.sqrt(np.mean(np.sum(psi * psi, axis=-1)))
    if rms > 0:  # a 2^3 lattice carries no displacement (only Nyquist modes): it stays a lattice
        psi *= rms_disp / rms
    g = np.arange(n) + 0.5
    zz, yy, xx = np.meshgrid(g, g, g, indexing="ij")
    base = np.stack([xx, yy, zz], axis=-1)
    pos = np.mod(base + psi, n).reshape(-1, 3)
    vel = psi.reshape(-1, 3).astype(np.float32)
    return pos, vel, delta


def zeldovich_box(m: int, box: float, rms_disp: float, seed: int, slope: float = -2.0):
    """An m^3 lattice in a periodic box of side ``box`` fine cells, displaced by the Zel'dovich
    field of a P ~ k^slope Gaussian delta on the m^3 lattice, rms |Psi| = rms_disp fine cells.
    Returns (pos float64[m^3,3] in [0,box), vel float32[m^3,3] = Psi in fine cells)."""
    pos, vel, _ = zeldovich_lattice(m, rms_disp * m / box, seed, slope)
    scale = box / m
    return np.mod(pos * scale, box), (vel * scale).astype(np.float32)


def lognormal_poisson(n: int, sigma: float, seed: int, mean_per_cell: float = 1.0,
                      slope: float = -2.0):
    """Poisson sample of a lognormal density on an n^3 fine grid.

    rho ~ exp(G - sigma^2/2), G Gaussian with P ~ k^slope normalised to std sigma;
    counts ~ Poisson(rho * mean_per_cell * n^3 / sum(rho)); positions uniform in the cell.
    Returns (pos float64[N,3], vel float32[N,3], counts int array [z,y,x]).
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    g = gaussian_field(n, slope, rng) * sigma
    rho = np.exp(g - 0.5 * sigma * sigma)
    lam = rho * (mean_per_cell * n ** 3 / rho.sum())
    counts = rng.poisson(lam)
    total = int(counts.sum())
    flat = counts.reshape(-1)
    cell = np.repeat(np.arange(flat.size, dtype=np.int64), flat)
    cz, rem = np.divmod(cell, n * n)
    cy, cx = np.divmod(rem, n)
    pos = np.stack([cx, cy, cz], axis=-1).astype(np.float64)
    pos += rng.random((total, 3))
    pos = np.mod(pos, n)
    vel = (0.05 * rng.standard_normal((total, 3))).astype(np.float32)
    return pos, vel, counts


def uniform_random(npart: int, box: float, seed: int):
    """Uniform random positions in [0, box)^3 (small test inputs)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    pos = rng.random((npart, 3)) * box
    vel = (0.05 * rng.standard_normal((npart, 3))).astype(np.float32)
    return pos, vel
