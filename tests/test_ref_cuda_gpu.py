"""The kick against the reference's own CUDA path.

``pm3_fft_cuda.cu`` and ``pp_force_kernel.cu`` are compiled from the reference
sources for sm_100a (oracle/build_ref.py) and called through their own C ABI
(oracle.RefCuda).  The reference PM3 (pm3_fft_cuda.cu:516-620) leaves its
velocity change in the shared device accumulator of pp_force_kernel.cu:496-547;
it is read back with c_gpu_velocity_get (pp_force_kernel.cu:515-522).  Its PP
(pp_force_kernel.cu:960-1050) then adds its own change and merges both into the
host velocities, as kick.f90:143-205 calls them.

Compared on the same inputs, in the reference's per-subtile mesh geometry
(CUBE_PM3_SUBTILE, Green tables from the caller, levels uniform and mixed):
* this library's PM3 velocity change, f2max and particle counts;
* the CPU restatement of the Fortran PM3 (oracle/pm3_oracle.c);
* the whole kick (PM3 then PP; and cube_kick_fine), f2max and vmax of PP;
* PM2 on a one-coarse-cell tile buffer, which is the reference PM3's mesh of a
  tile with one subtile per tile and ratio_sf = 1.

Bars: velocity changes within 1e-5 relative rms, f2max and vmax within 1e-5,
particle counts exact.  The velocities start at zero, so the final velocities
are the kick's velocity change.
"""
import dataclasses

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

SIXPI = float(np.float32(6 * np.pi))
TOL = 1e-5
APM3F = 3.5  # PM3 softening in mesh cells of the reference's defaults (parameters.f90:39)


def _rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


_IMAGES = {}
_GREENS = {}
_REFS = {}


def _image(case):
    """(image with zero velocities, GPU build name)."""
    if case not in _IMAGES:
        from cube2_b200 import ic
        from cube2_b200.layout import Layout, build_image
        from oracle.layouts import LAYOUTS
        if case in ("t32", "t32_edge", "t32b_edge"):
            img, _ = load_golden(case)
            build = "t32b" if case == "t32b_edge" else "t32"
        elif case == "zeldovich64":
            from cube2_b200 import workloads
            img = workloads.make("zeldovich64")
            build = "cfg0"
        elif case == "clumpy64":
            img = build_image(*ic.lognormal_poisson(64, 1.5, 4100)[:2], Layout(**LAYOUTS["cfg0"]))
            build = "cfg0"
        elif case == "clumpy96":
            img = build_image(*ic.lognormal_poisson(96, 1.5, 4200)[:2], Layout(**LAYOUTS["c96"]))
            build = "c96"
        else:
            raise KeyError(case)
        _IMAGES[case] = (dataclasses.replace(img, vp=np.zeros_like(img.vp)), build)
    return _IMAGES[case]


_CURRENT = []


def _ref(build):
    """The reference build; the previous one releases its workspace (about 2 GB of pinned host
    staging, pp_force_kernel.cu:372-373) when another build takes over."""
    from oracle.oracle import RefCuda
    if _CURRENT and _CURRENT[0] != build:
        _REFS[_CURRENT[0]].finalize()
    _CURRENT[:] = [build]
    if build not in _REFS:
        _REFS[build] = RefCuda(build)
    return _REFS[build]


def _greens(L, levels):
    """Green_3D(nft, apm3f, apm2f = 3.5 ratio_sf, 1 / ratio_sf) per level (initialize.f90:142-168)."""
    from cube2_b200.layout import RATIO_SF
    from oracle import oracle as O
    out = {}
    for lev in levels:
        rsf = int(RATIO_SF[lev - 1])
        nft = L.ntt * L.ratio_cs * rsf + 2 * L.ratio_cs * rsf
        key = (nft, rsf)
        if key not in _GREENS:
            _GREENS[key] = O.green(nft, APM3F, 3.5 * rsf, 1.0 / rsf)
        out[lev] = _GREENS[key]
    return out


def _tables(L, mixed):
    from cube2_b200.layout import RATIO_SF, apm3_table, ixyz3_table
    ires = np.full(L.ns3, 2, np.int32)
    if mixed:
        ires[::3] = 3
    isort = np.arange(1, L.ns3 + 1, dtype=np.int32)
    return isort, ires, ixyz3_table(L), apm3_table(APM3F), RATIO_SF.copy()


_RUNS = {}


def _run(case, mixed):
    """The reference's kick and this library's, on the same image and tables."""
    key = (case, mixed)
    if key not in _RUNS:
        from cube2_b200.kick import CUBE_PM3_SUBTILE, FineKick
        img, build = _image(case)
        L = img.layout
        isort, ires, ix, apm3, rsf = _tables(L, mixed)
        greens = _greens(L, sorted(set(ires.tolist())))
        ref = _ref(build).kick(img, isort, ires, ix, apm3, rsf, greens, 1.0, SIXPI, 1.0)
        fk = FineKick(L, pm3_mode=CUBE_PM3_SUBTILE, apm3f=APM3F)
        vp1, f2, vmax, pt = fk.c_pm3_force_kernel(img, isort, ires, ix, rsf, 1.0, SIXPI, 1.0, greens=greens)
        vp2, f2p, vmaxp, ptp, _ = fk.c_pp_force_kernel(img, isort, ires, ix, apm3, rsf, 1.0, SIXPI, 1.0,
                                                       vp=vp1.copy())
        vpk, out = fk.kick_fine(img, isort, ires, ix, apm3, rsf, 1.0, SIXPI, 1.0, greens=greens)
        _RUNS[key] = dict(img=img, ref=ref, pm3=(vp1, f2, vmax, pt), pp=(vp2, f2p, vmaxp, ptp), fine=(vpk, out),
                          tables=(isort, ires, ix, apm3, rsf), greens=greens)
    return _RUNS[key]


CASES = [("t32", False), ("t32", True), ("t32_edge", False), ("t32b_edge", False), ("t32b_edge", True),
         ("zeldovich64", False), ("clumpy64", False), ("clumpy64", True), ("clumpy96", False)]


@pytest.mark.parametrize("case,mixed", CASES)
def test_pm3_matches_reference_cuda(gpu, case, mixed):
    r = _run(case, mixed)
    img, ref = r["img"], r["ref"]
    vp1, f2, _, pt = r["pm3"]
    act = img.active
    dv_ref = ref["dv_pm3"]
    assert np.sum(dv_ref[act].astype(np.float64) ** 2) > 0
    assert _rel_rms(vp1[act], dv_ref[act]) < TOL
    # neither kicks the buffer copies
    assert np.all(dv_ref[~act] == 0) and np.all(vp1[~act] == 0)
    assert abs(f2 - ref["f2max_pm3"]) <= TOL * ref["f2max_pm3"]
    np.testing.assert_array_equal(pt, ref["ptotal_pm3"])


@pytest.mark.parametrize("case,mixed", CASES)
def test_kick_matches_reference_cuda(gpu, case, mixed):
    r = _run(case, mixed)
    img, ref = r["img"], r["ref"]
    act = img.active
    vp2, f2p, vmaxp, ptp = r["pp"]
    assert _rel_rms(vp2[act], ref["vp"][act]) < TOL
    assert np.all(ref["vp"][~act] == 0) and np.all(vp2[~act] == 0)
    assert abs(f2p - ref["f2max_pp"]) <= TOL * ref["f2max_pp"]
    np.testing.assert_allclose(vmaxp, ref["vmax"], rtol=TOL)
    np.testing.assert_array_equal(ptp, ref["ptotal_pp"])
    # the whole kick in one call: PM3 and PP f2max, vmax after the kick
    vpk, out = r["fine"]
    assert _rel_rms(vpk[act], ref["vp"][act]) < TOL
    assert abs(out[0] - ref["f2max_pm3"]) <= TOL * ref["f2max_pm3"]
    assert abs(out[1] - ref["f2max_pp"]) <= TOL * ref["f2max_pp"]
    np.testing.assert_allclose(out[2:], ref["vmax"], rtol=TOL)


@pytest.mark.parametrize("case,mixed", [("t32", False), ("t32", True), ("t32_edge", False), ("t32b_edge", True),
                                        ("clumpy64", False)])
def test_pm3_restatement_matches_reference_cuda(gpu, case, mixed):
    """The CPU restatement of the Fortran PM3 (kick.f90:403-568) against the reference CUDA PM3:
    the checker that the periodic geometry's PM3 tests use is itself pinned here."""
    from cube2_b200.layout import RATIO_SF
    from oracle import oracle as O
    r = _run(case, mixed)
    img, ref = r["img"], r["ref"]
    isort, ires, ix, apm3, rsf = r["tables"]
    want = O.pm3_subtile(img, ires, ix, RATIO_SF, r["greens"], 1.0, SIXPI, 1.0)
    act = img.active
    assert _rel_rms(ref["dv_pm3"][act], want["vp"][act]) < TOL
    assert abs(want["f2max"] - ref["f2max_pm3"]) <= TOL * ref["f2max_pm3"]


def test_pm2_matches_reference_cuda_mesh(gpu):
    """PM2 (pm_thread with kick.f90:77-105's parameters) on a one coarse-cell tile buffer solves
    one mesh of (nt + 2) ratio_cs points per tile with Green_3D(ngt, apm2, apm1, 1): the mesh the
    reference CUDA PM3 builds for a tile that is a single subtile at ratio_sf = 1
    (pm3_fft_cuda.cu:402-404).  The reference PM3 with that table is compared with this
    library's PM2."""
    from cube2_b200 import ic
    from cube2_b200 import longrange as LR
    from cube2_b200.layout import Layout, apm3_table, build_image, ixyz3_table
    from oracle import oracle as O
    L = Layout(ng=32, nnt=2, nns=2, ratio_cs=4, ngb=4, app=0.1)
    pos, vel = ic.uniform_random(3000, 32.0, 13)
    img = build_image(pos, np.zeros_like(vel), L)
    vp, f2, _ = LR.pm2_force(img, 3.5, 14.0, 1.0, SIXPI, 1.0)
    L1 = Layout(ng=32, nnt=2, nns=1, ratio_cs=4, ngb=4, app=0.1)
    img1 = dataclasses.replace(img, layout=L1)
    ngt = L.nte * L.ratio_cs
    G = O.green(ngt, 3.5, 14.0, 1.0)
    ones = np.ones(7, np.int32)
    ref = _ref("t32s1").kick(img1, np.arange(1, L1.ns3 + 1, dtype=np.int32), np.full(L1.ns3, 2, np.int32),
                             ixyz3_table(L1), apm3_table(APM3F), ones, {2: G}, 1.0, SIXPI, 1.0)
    act = img.active
    assert np.sum(ref["dv_pm3"][act].astype(np.float64) ** 2) > 0
    assert _rel_rms(vp[act], ref["dv_pm3"][act]) < TOL
    assert abs(f2 - ref["f2max_pm3"]) <= TOL * ref["f2max_pm3"]
