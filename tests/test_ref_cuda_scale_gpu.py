"""The kick at the bench's scale against the reference's own CUDA path, compared and timed.

clustered256 (the bench's image: 16.8 M particles of a sigma = 1.5 lognormal density, 2^3
tiles, 20.2 M stored with their buffers) in the reference's per-subtile mesh geometry
(CUBE_PM3_SUBTILE, every subtile at ratio_sf = 2, Green tables from the caller), through both
C ABIs on the same pinned host arrays:

* parity: the PM3 velocity change (read from the reference's device accumulator,
  pp_force_kernel.cu:515-522), the whole kick (PM3 then PP), f2max, vmax and the particle
  counts, at the bars of test_ref_cuda_gpu (1e-5 relative rms, counts exact);
* timing: wall clock of c_pm3_force_kernel and of c_pp_force_kernel (each returns with its
  results in the caller's host arrays) for the reference build and for this library, and of
  this library's single-call cube_kick_fine, after one warm-up kick each, median of three
  (the calls interleaved).  The figures are printed, and written as JSON to the file that
  CUBE_REF_TIMING_JSON names when it is set.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIXPI = float(np.float32(6 * np.pi))
TOL = 1e-5
APM3F = 3.5  # PM3 softening in mesh cells of the reference's defaults (parameters.f90:39)


def _rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def _pinned_image(img):
    """The image with its arrays in page-locked host memory (numpy views of pinned tensors)."""
    import dataclasses

    import torch

    def pin(a):
        return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()

    return dataclasses.replace(img, xp=pin(img.xp), vp=pin(np.zeros_like(img.vp)), rhoc=pin(img.rhoc),
                               idx_b_r=pin(img.idx_b_r))


@pytest.mark.timeout(1200)
def test_clustered256_against_reference_cuda(gpu):
    import torch

    from cube2_b200 import workloads as W
    from cube2_b200.kick import CUBE_PM3_SUBTILE, FineKick
    from cube2_b200.layout import RATIO_SF, apm3_table, ixyz3_table
    from oracle import oracle as O

    img = _pinned_image(W.make("clustered256"))
    L = img.layout
    isort = np.arange(1, L.ns3 + 1, dtype=np.int32)
    ires = np.full(L.ns3, 2, np.int32)
    ix, apm3, rsf = ixyz3_table(L), apm3_table(APM3F), RATIO_SF.copy()
    nft = L.ntt * L.ratio_cs * 2 + 2 * L.ratio_cs * 2
    greens = {2: O.green(nft, APM3F, 3.5 * 2, 0.5)}
    ref = O.RefCuda("cfg1")
    fk = FineKick(L, pm3_mode=CUBE_PM3_SUBTILE, apm3f=APM3F)
    try:
        # parity: both kicks from zero velocities
        r = ref.kick(img, isort, ires, ix, apm3, rsf, greens, 1.0, SIXPI, 1.0)
        vp1, f2, _, pt = fk.c_pm3_force_kernel(img, isort, ires, ix, rsf, 1.0, SIXPI, 1.0, greens=greens)
        vp2, f2p, vmaxp, ptp, _ = fk.c_pp_force_kernel(img, isort, ires, ix, apm3, rsf, 1.0, SIXPI, 1.0,
                                                       vp=vp1.copy())
        act = img.active
        e_pm3 = _rel_rms(vp1[act], r["dv_pm3"][act])
        e_kick = _rel_rms(vp2[act], r["vp"][act])
        assert e_pm3 < TOL and e_kick < TOL
        assert np.all(vp2[~act] == 0) and np.all(r["vp"][~act] == 0)
        assert abs(f2 - r["f2max_pm3"]) <= TOL * r["f2max_pm3"]
        assert abs(f2p - r["f2max_pp"]) <= TOL * r["f2max_pp"]
        np.testing.assert_allclose(vmaxp, r["vmax"], rtol=TOL)
        np.testing.assert_array_equal(pt, r["ptotal_pm3"])
        np.testing.assert_array_equal(ptp, r["ptotal_pp"])

        # timing on the same pinned arrays; vp is kicked in place, its values do not matter
        vp = img.vp
        args = (isort, ires, ix, apm3, rsf)

        def ref_call():
            return ref.kick_wall(img, *args, greens, 1.0, SIXPI, 1.0, vp)

        def ours_two_calls():
            import time
            t0 = time.perf_counter()
            fk.c_pm3_force_kernel(img, isort, ires, ix, rsf, 1.0, SIXPI, 1.0, greens=greens, vp=vp)
            t1 = time.perf_counter()
            fk.c_pp_force_kernel(img, *args, 1.0, SIXPI, 1.0, vp=vp)
            return t1 - t0, time.perf_counter() - t1

        def ours_one_call():
            import time
            t0 = time.perf_counter()
            fk.kick_fine(img, *args, 1.0, SIXPI, 1.0, greens=greens, vp=vp)
            return time.perf_counter() - t0

        ref_call(), ours_two_calls(), ours_one_call()  # warm-up (workspaces, plans, PP shape tuning)
        tr, to, tf = [], [], []
        for _ in range(3):
            tr.append(ref_call())
            to.append(ours_two_calls())
            tf.append(ours_one_call())
        torch.cuda.synchronize()
        med = lambda v: float(np.median(v)) * 1e3  # noqa: E731
        res = {
            "workload": "clustered256", "geometry": "per-subtile buffered meshes (CUBE_PM3_SUBTILE), ratio_sf 2",
            "particles": int(img.n_particles), "stored": int(img.n_used),
            "host_arrays": "pinned", "timing": "wall clock per call, median of 3 after 1 warm-up",
            "reference_cuda_ms": {"c_pm3_force_kernel": med([t[0] for t in tr]),
                                  "c_pp_force_kernel": med([t[1] for t in tr]),
                                  "kick": med([t[0] + t[1] for t in tr])},
            "library_ms": {"c_pm3_force_kernel": med([t[0] for t in to]),
                           "c_pp_force_kernel": med([t[1] for t in to]),
                           "kick": med([t[0] + t[1] for t in to]), "cube_kick_fine": med(tf)},
            "parity": {"pm3_rel_rms": e_pm3, "kick_rel_rms": e_kick},
        }
        print(json.dumps(res))
        out = os.environ.get("CUBE_REF_TIMING_JSON")
        if out:
            with open(out, "w") as f:
                json.dump(res, f, indent=1)
    finally:
        ref.finalize()
