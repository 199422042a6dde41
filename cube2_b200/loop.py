"""Kick-drift time loop of one image on the device (the reference's main loop, main.f90:20-52:
drift, buffer_grid, buffer_x, kick, buffer_v per step), with Zel'dovich initial conditions
built on the device.

The initial image is a lattice with one particle at the centre of every fine cell, stored in
the reference layout with its periodic buffers; one drift with vp = Psi and dt_mid = 1 then
moves every particle by its Zel'dovich displacement Psi (fine cells) through the library's own
fixed-point drift, so the initial offsets are exactly what the reference's drift would write.
torch is used for device memory and for the Gaussian field's FFTs (input generation only).
"""
from __future__ import annotations

import numpy as np

from .drift import DeviceImage
from .kick import CUBE_PM3_PERIODIC, FineKick
from .layout import RATIO_SF, Image, Layout, apm3_table, ixyz3_table


def gaussian_field_device(n: int, slope: float, seed: int, device):
    """Real Gaussian field on n^3 with P(k) ~ k^slope (k != 0), zero mean, unit variance; and its
    transform (for the displacement)."""
    import torch
    g = torch.Generator(device=device).manual_seed(seed)
    white = torch.randn((n, n, n), generator=g, device=device, dtype=torch.float32)
    wk = torch.fft.rfftn(white)
    del white
    k1 = torch.fft.fftfreq(n, d=1.0 / n, device=device)
    kr = torch.fft.rfftfreq(n, d=1.0 / n, device=device)
    k2 = k1[:, None, None] ** 2 + k1[None, :, None] ** 2 + kr[None, None, :] ** 2
    amp = torch.where(k2 > 0, k2.clamp(min=1e-30) ** (slope / 4.0), torch.zeros_like(k2))
    wk *= amp
    wk[0, 0, 0] = 0
    f = torch.fft.irfftn(wk, s=(n, n, n))
    sd = f.std()
    return f / sd, wk / sd, k1, kr


def zeldovich_displacement_device(n: int, rms_disp: float, seed: int, device, slope: float = -2.0,
                                  clip: float | None = None):
    """Psi [z][y][x][3] (components x, y, z) of the Zel'dovich field of a P ~ k^slope Gaussian
    delta on the n^3 lattice, rms |Psi| = rms_disp lattice cells."""
    import torch
    _, dk, k1, kr = gaussian_field_device(n, slope, seed, device)
    k2 = k1[:, None, None] ** 2 + k1[None, :, None] ** 2 + kr[None, None, :] ** 2
    k2[0, 0, 0] = 1.0
    comps = []
    for kc in (kr[None, None, :], k1[None, :, None], k1[:, None, None]):  # x, y, z
        comps.append(torch.fft.irfftn(1j * kc * dk / k2 * (n / (2 * np.pi)), s=(n, n, n)).float())
    del dk
    psi = torch.stack(comps, dim=-1)
    del comps
    rms = torch.sqrt(torch.mean(torch.sum(psi.double() ** 2, dim=-1)))
    psi *= float(rms_disp / rms)
    if clip is not None:
        psi.clamp_(-clip, clip)
    return psi


def lattice_image_device(L: Layout, values, device) -> DeviceImage:
    """One particle at the centre of every fine cell (ng^3 particles), stored with the
    periodic buffers of layout L; vp of every stored copy = values[fine z, y, x] (a [ng]^3 x 3
    device tensor).  pid = (z * ng + y) * ng + x of the fine cell."""
    import torch
    r = L.ratio_cs
    per = r ** 3
    nte, ncb, nt, nnt, nc, ng = L.nte, L.ncb, L.nt, L.nnt, L.nc, L.ng
    ncell = nnt ** 3 * nte ** 3
    n_used = ncell * per
    img = Image(L, np.zeros((0, 3), np.int16), np.zeros((0, 3), np.float32),
                np.full((nnt, nnt, nnt, nte, nte, nte), per, np.int32),
                (np.arange(1, nnt ** 3 * nte * nte + 1, dtype=np.int64) * nte * per).reshape(nnt, nnt, nnt, nte, nte),
                np.zeros(0, np.int64), np.zeros(0, bool), n_particles=ng ** 3)
    di = DeviceImage(img, device, headroom=1.0, with_pid=True)
    cap = int(n_used * 1.05) + 1024
    di.xp = torch.zeros((cap, 3), dtype=torch.int16, device=device)
    di.vp = torch.zeros((cap, 3), dtype=torch.float32, device=device)
    di.pid = torch.zeros((cap,), dtype=torch.int64, device=device)
    di.cap = cap
    di.n_used = n_used
    chunk = 1 << 24
    for q0 in range(0, n_used, chunk):
        q = torch.arange(q0, min(q0 + chunk, n_used), device=device, dtype=torch.int64)
        E, f = q // per, q % per
        fd = torch.stack([f % r, (f // r) % r, f // (r * r)], dim=1)
        u = fd * (65536 // r) + 32768 // r
        di.xp[q0:q0 + q.numel()] = torch.where(u >= 32768, u - 65536, u).to(torch.int16)
        t, rem = E // nte ** 3, E % nte ** 3
        c = torch.stack([rem % nte, (rem // nte) % nte, rem // (nte * nte)], dim=1)
        tt = torch.stack([t % nnt, (t // nnt) % nnt, t // (nnt * nnt)], dim=1)
        gcell = torch.remainder(tt * nt + c - ncb, nc)
        fine = gcell * r + fd
        di.vp[q0:q0 + q.numel()] = values[fine[:, 2], fine[:, 1], fine[:, 0]]
        di.pid[q0:q0 + q.numel()] = (fine[:, 2] * ng + fine[:, 1]) * ng + fine[:, 0]
    return di


def uniform_tables(L: Layout, apm3f: float):
    """(isort, ires, ixyz3, apm3, ratio_sf) of a kick with every subtile at level 2 (ratio_sf 2)."""
    return (np.arange(1, L.ns3 + 1, dtype=np.int32), np.full(L.ns3, 2, np.int32), ixyz3_table(L),
            apm3_table(apm3f), RATIO_SF.copy())


def zeldovich_start(L: Layout, rms_disp: float, seed: int, vfac: float, device) -> DeviceImage:
    """Zel'dovich initial conditions on the device: lattice + one drift by Psi, then vp = vfac Psi."""
    import torch
    psi = zeldovich_displacement_device(L.ng, rms_disp, seed, device, clip=0.95 * L.ncb * L.ratio_cs)
    di = lattice_image_device(L, psi, device)
    del psi
    torch.cuda.synchronize()
    FineKick(L, pm3_mode=CUBE_PM3_PERIODIC).configure()
    vz = float(di.vp[:di.n_used, 2].abs().max().item())
    di.drift(1.0, vz)
    di.vp[:di.n_used] *= vfac
    return di


def positions_by_pid(di: DeviceImage):
    """Physical positions (fine cells, float64) of every particle, indexed by pid (device tensor)."""
    import torch
    L = di.layout
    nte, ncb, nt, nnt = L.nte, L.ncb, L.nt, L.nnt
    counts = di.rhoc.to(torch.int64)
    cell = torch.repeat_interleave(torch.arange(counts.numel(), device=counts.device), counts)
    t, rem = cell // nte ** 3, cell % nte ** 3
    c = torch.stack([rem % nte, (rem // nte) % nte, rem // (nte * nte)], dim=1)
    phys = ((c >= ncb) & (c < ncb + nt)).all(dim=1)
    tt = torch.stack([t % nnt, (t // nnt) % nnt, t // (nnt * nnt)], dim=1)
    n = di.n_used
    u = di.xp[:n].to(torch.int32) & 0xFFFF
    pos = ((tt * nt + c - ncb).double() + (u.double() + 0.5) / 65536.0) * L.ratio_cs
    out = torch.zeros((L.ng ** 3, 3), dtype=torch.float64, device=pos.device)
    out[di.pid[:n][phys]] = pos[phys]
    return out


def rms_position_difference(a: DeviceImage, b: DeviceImage) -> float:
    """rms over particles of the periodic distance between their positions in two images (fine cells)."""
    import torch
    pa, pb = positions_by_pid(a), positions_by_pid(b)
    box = float(a.layout.ng)
    d = torch.remainder(pa - pb + box / 2, box) - box / 2
    return float(torch.sqrt(torch.mean(torch.sum(d * d, dim=1))).item())


SIXPI = float(np.float32(6 * np.pi))


def physical_mask(di: DeviceImage):
    """Per stored copy (device bool tensor): does it lie in its tile's physical region?"""
    import torch
    L = di.layout
    nte, ncb, nt = L.nte, L.ncb, L.nt
    e = torch.arange(nte, device=di.rhoc.device) - ncb
    inner1 = (e >= 0) & (e < nt)
    inner = (inner1[:, None, None] & inner1[None, :, None] & inner1[None, None, :]).reshape(-1).repeat(L.nnt ** 3)
    return torch.repeat_interleave(inner, di.rhoc.to(torch.int64))


def growth_rate(di: DeviceImage, apm3f: float, stream=None) -> float:
    """c of the linear growing mode F = c Psi on the initial image, whose velocities are still
    Psi: one kick with coefficient 1 applied to a copy of the velocities, and the regression of
    the force on Psi over the physical particles."""
    import torch
    L = di.layout
    fk = FineKick(L, pm3_mode=CUBE_PM3_PERIODIC, apm3f=apm3f)
    n = di.n_used
    psi = di.vp[:n].clone()
    out = torch.zeros(8, device=di.vp.device)
    fk.kick_fine_device(di.rhoc, di.idx, di.xp, n, di.vp, out, *uniform_tables(L, apm3f), 1.0, SIXPI, 1.0,
                        stream=stream)
    torch.cuda.synchronize()
    force = (di.vp[:n] - psi).double()
    di.vp[:n] = psi
    m = physical_mask(di)
    p = psi.double()[m]
    return float((force[m] * p).sum().item() / (p * p).sum().item())


class TimeLoop:
    """drift (+ buffer_grid, buffer_x), kick, buffer_v per step (main.f90:26-31) on a device image,
    with a fixed step: the kick adds coef * force to vp, the drift moves by dt_mid * vp.  The
    kick is the plain split (PM3 softened at apm3f mesh cells + PP within apm3f / 2 fine cells)
    or, with a learned shell, the cutoff-1 split plus the shell's force."""

    def __init__(self, di: DeviceImage, apm3f: float, coef: float, dt_mid: float, shell=None, shell_scale: float = 1.0,
                 stream=None):
        import torch
        self.di = di
        self.fk = FineKick(di.layout, pm3_mode=CUBE_PM3_PERIODIC, apm3f=apm3f)
        self.tabs = uniform_tables(di.layout, apm3f)
        self.coef = float(coef)
        self.dt_mid = float(dt_mid)
        self.shell, self.shell_scale = shell, float(shell_scale)
        self.stream = stream
        self.out = torch.zeros(8, device=di.vp.device)
        self.vz = float(di.vp[:di.n_used, 2].abs().max().item())

    def step(self, events=None):
        """One step; `events` (three CUDA events) are recorded on the loop's stream before the
        drift, between drift and kick, and after buffer_v."""
        di = self.di
        self.fk.configure()
        st = self.stream
        if events:
            events[0].record(st) if st is not None else events[0].record()
        di.drift(self.dt_mid, self.vz, self.stream)
        if events:
            events[1].record(st) if st is not None else events[1].record()
        self.fk.kick_fine_device(di.rhoc, di.idx, di.xp, di.n_used, di.vp, self.out, *self.tabs, 1.0, SIXPI,
                                 self.coef, stream=self.stream)
        if self.shell is not None:
            self.shell.kick(di.rhoc, di.idx, di.xp, di.n_used, di.vp, self.shell_scale, SIXPI, self.coef,
                            stream=self.stream)
        di.buffer_v(self.stream)
        if events:
            events[2].record(st) if st is not None else events[2].record()
        import torch
        if st is not None:
            st.synchronize()  # out is read on the host below
        else:
            torch.cuda.synchronize()  # the library's own stream
        self.vz = float(self.out[4].item())  # vmax_z after the kick: nlayer of the next drift

    def error_word(self) -> int:
        import torch
        return int(self.out[5:6].cpu().view(torch.int32).item())


def clone_image(di: DeviceImage) -> DeviceImage:
    """A second device image with the same contents (its own arrays)."""
    import copy
    c = copy.copy(di)
    n = di.n_used
    c.rhoc, c.idx = di.rhoc.clone(), di.idx.clone()
    c.xp, c.vp = di.xp.clone(), di.vp.clone()
    c.pid = None if di.pid is None else di.pid.clone()
    c._spare = None
    c.n_used = n
    return c


def start_with_growth(L: Layout, rms_disp: float, seed: int, growth_per_step: float, apm3f: float, device):
    """Zel'dovich start in the linear growing mode: (image with vp = sqrt(c) Psi, step dt, c)."""
    di = zeldovich_start(L, rms_disp, seed, 1.0, device)
    c = growth_rate(di, apm3f)
    if not c > 0:
        raise RuntimeError(f"no growing mode: c = {c}")
    dt = float(np.log1p(growth_per_step) / np.sqrt(c))
    di.vp[:di.n_used] *= float(np.sqrt(c))
    return di, dt, c


def snapshots(L: Layout, rms_disp: float, seed: int, growth_per_step: float, apm3f: float, steps: int,
              every: int, device):
    """Host images of a plain loop on layout L taken every `every` steps (step 0 included): the
    method's own snapshots, for training the learned shell."""
    di, dt, _ = start_with_growth(L, rms_disp, seed, growth_per_step, apm3f, device)
    loop = TimeLoop(di, apm3f, coef=dt, dt_mid=dt)
    out = [di.to_host()]
    for k in range(1, steps + 1):
        loop.step()
        if k % every == 0:
            out.append(di.to_host())
    return out
