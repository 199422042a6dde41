#!/usr/bin/env python
"""Benchmark of the fine-scale kick (PM3 + PP) on B200.

One step = one full fine-scale kick (PM3 fine-mesh force + PP short-range
force + velocity update) over the whole image of the chosen workload
(default ``clustered256``: ~16.8M clustered particles, 512^3 PM3 mesh, PP
cutoff 2 fine cells; see cube2_b200/workloads.py).

* ``value``   particle kicks/s with the inputs resident in HBM
  (cube_kick_fine_device), K steps timed with CUDA events on the launching
  stream, max over ranks; every rank runs its own replica (the kick of one
  image runs on one GPU; N > 1 = independent replicas).
* ``e2e``     the same metric through the host C-ABI (cube_kick_fine) with
  pinned host buffers: every step uploads xp/vp/rhoc/idx_b_r and downloads vp.
* ``roofline`` the PP force kernel (FP32 CUDA cores): 38 FLOP per accepted
  ordered pair (pairs counted for this input) / its average launch time,
  against the FP32 FMA peak measured in the same run.
* ``cpu_baseline`` / ``--impl reference``: the reference's own CPU PP kernel
  (pp_force_kernel.c, built from the reference sources into oracle/_ref) plus
  the CPU restatement of the reference PM3 on the same inputs, a full kick of
  the whole image per step.
* ``batch``   the batched uneven boxes (batch512) in one kick, as a CUDA graph
  and against one kick call per box; ``conservation`` the FP64 momentum and
  kinetic-energy change of one kick; ``drift`` and ``learned`` the other legs;
  ``loop`` the 20-step kick-drift loop of 512^3 particles on a 1024^3 mesh
  (loop512), plain and with the learned shell (``--no-loop`` skips it).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "particle kicks/s (PM3+PP) on 1 B200, learned vs plain at equal rms force error"
UNIT = "particle-kicks/s"
PP_FLOP_PER_PAIR = 38  # 3 sub, 5 r^2, rsqrt, 1/r^2, 2 ep, 18 polynomial+reciprocal, 1 diff, 1 scale, 6 accumulate
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one k_pp_force launch per stored
# particle, from an ncu capture on clustered192 (242.6 MB + 65.1 MB over 9,025,370 stored
# particles); the kernel streams the sorted particles and vp once per launch, so the figure is
# scaled to a full launch by the stored particle count
PP_DRAM_BYTES_PER_STORED = (242_559_488 + 65_138_432) / 9_025_370


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="clustered256")
    ap.add_argument("--truth-targets", type=int, default=10000)
    ap.add_argument("--no-truth", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-loop", action="store_true")
    return ap.parse_args()


def max_over_ranks(x: float, world: int, device) -> float:
    """The maximum of x over the ranks (each rank's device time; the job ends with the slowest)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(
        os.environ.get("LOCAL_RANK", "0"))


# ------------------------------------------------------------------------------------------------
# clocks during the timed region


class Clocks:
    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            # wait for the first sample, so that the sampler is running when the timed region starts
            first = self.proc.stdout.readline()
            if first:
                self.lines.append(first)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=10)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        return self.summarize(self.lines[1:] + out.splitlines(), self.uuid)  # the first sample predates the region

    @classmethod
    def summarize(cls, lines, uuid: str | None = None):
        """Median SM clock, max SM clock and the throttle reasons seen active, from the sampler's
        CSV lines (FIELDS order) of the GPU `uuid` (all GPUs when None); None without samples."""
        rows = []
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            if uuid and f[0] != uuid:
                continue
            rows.append(f)
        if not rows:
            return None

        def num(v):
            return v.replace(".", "", 1).isdigit()
        sm = [float(r[1]) for r in rows if num(r[1])]
        smax = max((float(r[2]) for r in rows if num(r[2])), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(rows)}


# ------------------------------------------------------------------------------------------------


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from cube2_b200 import workloads as W
    from cube2_b200.kick import CUBE_PM3_PERIODIC, CUBE_PM3_TILE_PERIODIC, FineKick, force_truth_fp64

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world > 1:
        dist.init_process_group("nccl", device_id=dev)
    w = W.WORKLOADS[args.workload]
    img = W.make(args.workload)
    L = img.layout
    isort, ires, ix, apm3, rs = W.tables(args.workload)
    batch = w["kind"] == "batch"  # independent periodic boxes, one PM3 mesh per parent tile
    fk = FineKick(L, pm3_mode=CUBE_PM3_TILE_PERIODIC if batch else CUBE_PM3_PERIODIC, apm3f=w["apm3f"])
    N = img.n_particles
    a_mid, dt = np.float32(6 * np.pi), np.float32(1.0)  # dv = force

    d_rhoc = torch.from_numpy(img.rhoc.reshape(-1).copy()).to(dev)
    d_idx = torch.from_numpy(img.idx_b_r.reshape(-1).copy()).to(dev)
    d_xp = torch.from_numpy(img.xp.reshape(-1).copy()).to(dev)
    vp0 = torch.from_numpy(img.vp.reshape(-1).copy()).to(dev)
    d_vp = vp0.clone()
    d_out = torch.zeros(8, dtype=torch.float32, device=dev)
    # a dedicated stream: the kernels and the timing events must share it
    stream = torch.cuda.Stream(dev)

    torch.cuda.synchronize()

    def kick():
        fk.kick_fine_device(d_rhoc, d_idx, d_xp, img.n_used, d_vp, d_out, isort, ires, ix, apm3, rs, 1.0, a_mid,
                            dt, stream=stream)

    # algorithmic work of the dominant kernel and the FP32 denominator
    pairs = fk.pp_pair_count(img, ires, ix, apm3, rs)
    fp32_peak = fk.fp32_peak_tflops()

    for _ in range(max(args.warmup, 0)):
        kick()
    torch.cuda.synchronize()
    err_word = int(d_out[5:6].cpu().view(torch.int32).item())
    if err_word:
        raise RuntimeError(f"device error mask {err_word}")
    fk.enable_timing(True)
    fk.timing_read()
    launches0 = fk.launch_count()
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    clocks = Clocks(uuid)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        kick()
    t1.record(stream)
    torch.cuda.synchronize()
    ck = clocks.stop()
    ms = t0.elapsed_time(t1)
    launches = fk.launch_count() - launches0
    stages = fk.timing_read()
    fk.enable_timing(False)
    ms = max_over_ranks(ms, world, dev)
    ms_step = ms / max(args.steps, 1)
    value = N * world * args.steps / (ms * 1e-3)

    # the PP kernel shape the autotuner picked during the warm-up (cube_pp_shapes)
    from cube2_b200.kick import pp_shapes
    table, cur = pp_shapes()
    pp_shape = {**{k: table[cur][k] for k in ("chunk", "jtile", "unroll", "blocks", "packed")}, "index": cur,
                "tuning_ms": [round(float(t["ms"]), 3) for t in table],
                "what": "autotuned on the first kick: work list + PP force kernel timed per shape"}

    # the same kick replayed as one captured CUDA graph (cube_kick_graph_*)
    graph = None
    try:
        kg = fk.kick_graph(d_rhoc, d_idx, d_xp, img.n_used, d_vp, d_out, isort, ires, ix, apm3, rs, 1.0, a_mid, dt)
        for _ in range(max(args.warmup, 0)):
            kg.launch(stream)
        torch.cuda.synchronize()
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(args.steps):
            kg.launch(stream)
        g1.record(stream)
        torch.cuda.synchronize()
        kg.close()
        gms = g0.elapsed_time(g1) / max(args.steps, 1)
        graph = {"ms_per_step": gms, "value": N / (gms * 1e-3), "unit": UNIT,
                 "what": "the device kick captured once as a CUDA graph and replayed per step"}
    except Exception as e:  # the graph is reported beside the main number, never instead of it
        graph = {"error": repr(e)}

    # e2e through the host C-ABI with pinned buffers
    e2e = None
    if not args.no_e2e:
        def pinned(a):
            t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
            return t.numpy()
        from cube2_b200.layout import Image
        himg = Image(L, pinned(img.xp), pinned(img.vp), pinned(img.rhoc), pinned(img.idx_b_r), img.pid, img.active,
                     N)
        vp_host = pinned(img.vp.copy())
        fk.kick_fine(himg, isort, ires, ix, apm3, rs, 1.0, a_mid, dt, vp=vp_host)  # warm
        if world > 1:
            dist.barrier()
        te = time.perf_counter()
        for _ in range(args.steps):
            fk.kick_fine(himg, isort, ires, ix, apm3, rs, 1.0, a_mid, dt, vp=vp_host)
        te = time.perf_counter() - te
        te = max_over_ranks(te, world, dev)
        h2d = img.xp.nbytes + img.vp.nbytes + img.rhoc.nbytes + img.idx_b_r.nbytes
        d2h = img.vp.nbytes + 24
        e2e = {"value": N * world * args.steps / te, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": 1e3 * te / args.steps}

    # FP64 momentum and kinetic-energy change of one kick, reduced on the device (outside the timed region)
    conservation = None
    try:
        from cube2_b200.kick import kick_sums
        d_vp.copy_(vp0)
        kick()
        torch.cuda.synchronize()
        c0 = torch.cuda.Event(enable_timing=True)
        c1 = torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        cs = kick_sums(d_rhoc, d_idx, img.n_used, vp0, d_vp, 1.0, stream=stream)
        c1.record(stream)
        torch.cuda.synchronize()
        conservation = {"momentum_change": [float(x) for x in cs["momentum"]],
                        "momentum_change_rel": [float(a / b) for a, b in zip(cs["momentum"], cs["momentum_scale"])],
                        "kinetic_energy_change": cs["kinetic_energy"], "particles": cs["particles"],
                        "ms": c0.elapsed_time(c1),
                        "what": "cube_kick_sums over the physical particles of one kick (PM3 + PP), FP64 on the "
                                "device; momentum_change_rel = sum m dv / sum |m dv| per axis"}
    except Exception as e:  # reported beside the kick, never instead of it
        conservation = {"error": repr(e)}

    # force error against the FP64 direct sum (outside the timed region)
    truth = None
    if not args.no_truth and rank == 0:
        d_vp.copy_(vp0 * 0)
        kick()
        torch.cuda.synchronize()
        v = d_vp.cpu().numpy().reshape(-1, 3).astype(np.float64)
        kick_coef = float(np.float32(a_mid * dt / np.float32(6.0))) / np.pi
        act = np.nonzero(img.active)[0]
        rng = np.random.default_rng(12345)
        samp = rng.choice(act, min(args.truth_targets, act.size), replace=False)
        t_tr = time.perf_counter()
        if batch:  # every box is its own periodic box: the truth is summed per box
            samp = np.sort(samp[:min(samp.size, 2000)])
            Ft = batch_truth(args.workload, img, samp, force_truth_fp64)
        else:
            pos = W.physical_positions(img)
            Ft = force_truth_fp64(pos, float(L.ng), L.app, img.pid[samp])
        t_tr = time.perf_counter() - t_tr
        F = v[samp] / kick_coef
        dF = np.linalg.norm(F - Ft, axis=1)
        Fm = np.linalg.norm(Ft, axis=1)
        truth = {"rms_rel": float(np.sqrt(np.sum(dF ** 2) / np.sum(Fm ** 2))),
                 "p99_rel": float(np.percentile(dF / np.maximum(Fm, 1e-30), 99)),
                 "targets": int(samp.size), "truth": "FP64 Ewald-split periodic direct sum", "seconds": t_tr}

    pm3_ms = float(np.mean(stages[:, 0])) if len(stages) else None
    ppb_ms = float(np.mean(stages[:, 1])) if len(stages) else None
    ppf_ms = float(np.mean(stages[:, 2])) if len(stages) else None
    flops = PP_FLOP_PER_PAIR * pairs
    achieved = flops / (ppf_ms * 1e-3) / 1e12 if ppf_ms else None
    roofline = {"kernel": "k_pp_force (PP pair force + kick)", "bound": "fp32", "achieved": achieved,
                "peak": fp32_peak, "unit": "TFLOP/s", "frac": (achieved / fp32_peak) if achieved else None,
                "peak_source": "FP32 FMA probe measured in this run (MEASURED_PEAKS.json has no FP32 figure)",
                "flops_per_launch": int(flops), "pairs_per_launch": int(pairs),
                "traffic": float(PP_DRAM_BYTES_PER_STORED * img.n_used),
                "traffic_source": "ncu DRAM bytes of k_pp_force on clustered192, scaled by stored particles"}

    # the whole kick against its roofline model: algorithmic bytes B = 64 B per particle + 66 B per
    # mesh point (binning 16, deposit 6, PP 12, gather 6, velocity 24 B per particle; deposit 4,
    # R2C 8, k-space 18, inverse transforms 24, gather 12 B per mesh point) and F = 38 FLOP per
    # accepted pair, each at its measured peak; frac = (B / BW + F / FP32) / time per kick
    n_mesh = (w["box"] * w["rsf"]) ** 3 * L.nnt ** 3 if batch else (L.ng * w["rsf"]) ** 3
    kick_bytes = 64.0 * N + 66.0 * n_mesh
    hbm_peak, hbm_src = measured_hbm_peak()
    t_model = kick_bytes / (hbm_peak * 1e9) + flops / (fp32_peak * 1e12)
    roofline_kick = {"bound": "hbm + fp32", "bytes": kick_bytes, "flops": float(flops),
                     "model_ms": 1e3 * t_model, "ms": ms_step, "frac": 1e3 * t_model / ms_step,
                     "peaks": {"hbm_gbs": hbm_peak, "hbm_source": hbm_src, "fp32_tflops": fp32_peak},
                     "what": "B / BW + F / FP32 over the kick's time: 64 B per particle + 66 B per mesh point, "
                             "38 FLOP per accepted PP pair"}

    loop = per_box_loop(args.workload, fk, img, stream, a_mid, dt, ms_step) if batch and rank == 0 else None
    if batch:
        fk.configure()
    batch_obj = None
    if not batch and rank == 0 and not args.no_batch:
        try:
            batch_obj = batch_leg("batch512", stream, args.steps, args.warmup)
        except Exception as e:  # reported beside the kick, never instead of it
            batch_obj = {"error": repr(e)}
        fk.configure()
    drift = None
    if rank == 0:
        try:
            drift = drift_leg(img, CUBE_PM3_TILE_PERIODIC if batch else CUBE_PM3_PERIODIC, stream, args.steps,
                              args.warmup)
        except Exception as e:  # reported beside the kick, never instead of it
            drift = {"error": repr(e)}
        fk.configure()
    learned = None
    if not batch and not args.no_learned and rank == 0:
        try:
            learned = learned_variant(args, img, (isort, ires, ix, apm3, rs), stream, truth, value, ms_step)
        except Exception as e:  # reported beside the plain number, never instead of it
            learned = {"error": repr(e)}
        fk.configure()

    loop_obj = None
    if not batch and rank == 0 and not args.no_loop:
        # the 20-step kick-drift loop of 512^3 particles (plain, and with the learned shell)
        try:
            loop_obj = loop_leg("loop512", 20, max(args.warmup, 3), dev, stream, ("learned",))
            loop_obj["what"] = ("drift + buffer_grid + buffer_x + kick + buffer_v per step on device-resident "
                                "arrays (cube_drift_device, cube_kick_fine_device); the learned variant's P(k) "
                                "against the plain loop's after the same steps")
        except Exception as e:  # reported beside the kick, never instead of it
            loop_obj = {"error": repr(e)}
        fk.configure()

    cpu = None
    if batch:
        cpu = {"unavailable": "the reference CPU baseline is timed on the single-image workloads"}
    elif rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_reference(args.workload, img)
        except Exception as e:  # the baseline must not hide our number
            cpu = {"error": repr(e)}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32 (int16 fixed-point positions, fp64 Green table)",
            "data": ("synthetic (512 seeded Zel'dovich boxes of uneven size; see cube2_b200/workloads.py)" if batch
                     else "synthetic (seeded lognormal Poisson sample; see cube2_b200/workloads.py)"),
            "config": {"workload": args.workload, "particles": N, "n_used_stored": img.n_used,
                       "pm3_mesh": (f"{w['box'] * w['rsf']}^3 per box x {L.nnt ** 3} boxes" if batch
                                    else L.ng * w["rsf"]),
                       "pp_cutoff_fine_cells": w["apm3f"] / w["rsf"],
                       "softening_fine_cells": L.app, "assignment": "TSC", "variant": "plain (no learned shell)",
                       "layout": L.as_dict(), "parallelism": f"replicas x{world}",
                       "l2": ("inputs larger than L2 (meshes 512 x 64^3 fp32 = 537 MB, particle arrays > 290 MB)"
                              if batch else "inputs larger than L2 (mesh 512^3 fp32 = 537 MB, particle arrays > 120 MB)")},
            "stages_ms": {"pm3": pm3_ms, "pp_binning_and_worklist": ppb_ms, "pp_force": ppf_ms,
                          "note": "the PP binning and work list run on a second stream beside PM3"},
            "roofline": roofline, "roofline_kick": roofline_kick, "force_error": truth, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": ck, "cpu_baseline": cpu, "graph": graph, "pp_shape": pp_shape, "drift": drift, "learned": learned,
            "conservation": conservation, "batch": batch_obj, "loop": loop_obj}
    if loop is not None:
        line["per_box_loop"] = loop
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


LEARNED_BOUND = 0.01  # rms force error bound of the learned shell against the FP64 truth


def measured_hbm_peak():
    """(GB/s, source) of the HBM copy bandwidth measured on this pool's B200s."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s (of fallback)"


DRIFT_BYTES_PER_COPY = 26  # xp 6 + vp 12 + pid 8 bytes per stored copy, read once and written once


def drift_leg(img, pm3_mode, stream, steps, warmup):
    """The other half of a time step on the bench image: drift + buffer rebuild
    (cube_drift_device) and buffer_v (cube_buffer_v_device), timed with CUDA events.  Each drift
    moves the fastest particle by 0.1 coarse cells."""
    import torch
    from cube2_b200.drift import DeviceImage
    from cube2_b200.kick import FineKick
    dev = torch.device("cuda", torch.cuda.current_device())
    FineKick(img.layout, pm3_mode=pm3_mode).configure()
    di = DeviceImage(img, dev)
    vmax = float(np.abs(img.vp).max())
    vz = float(np.abs(img.vp[:, 2]).max())
    dt_mid = 0.1 * img.layout.ratio_cs / max(vmax, 1e-6)
    n_in = di.n_used
    for _ in range(max(warmup, 1)):
        di.drift(dt_mid, vz, stream)
        di.buffer_v(stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        di.drift(dt_mid, vz, stream)
        di.buffer_v(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(steps, 1)
    moved = DRIFT_BYTES_PER_COPY * (n_in + di.n_used)
    peak, src = measured_hbm_peak()
    gbs = moved / (ms * 1e-3) / 1e9
    return {"ms_per_step": ms, "value": di.n_physical / (ms * 1e-3), "unit": "particle-drifts/s",
            "stored_copies_in": int(n_in), "stored_copies_out": int(di.n_used), "physical": int(di.n_physical),
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                         "peak_source": src,
                         "bytes": f"{DRIFT_BYTES_PER_COPY} B per stored copy read + written (xp, vp, pid)"},
            "what": "drift + buffer_grid + buffer_x + buffer_v (cube_drift_device + cube_buffer_v_device), "
                    "two host synchronisations per drift for the new sizes"}


def learned_variant(args, img, tables, stream, truth_plain, value_plain, ms_plain):
    """The learned-shell kick on the same image: cutoff 1 (PM3 softened at 1 fine cell, PP
    within 1 fine cell) plus the MLP, trained here on config-3-style boxes with the library's
    own kernels.  Timed like the plain kick; its error against the FP64 truth is checked on the
    same sampled particles, and above LEARNED_BOUND the kick falls back to the plain one."""
    import torch
    from cube2_b200 import learned as Ln
    from cube2_b200 import workloads as W
    from cube2_b200.kick import CUBE_PM3_PERIODIC, FineKick, force_truth_fp64
    from cube2_b200.layout import apm3_table
    dev = torch.device("cuda", torch.cuda.current_device())
    shell, scale, tinfo = Ln.train_shell(dev)
    # the learned kick on the bench image
    L = img.layout
    isort, ires, ix, _, rs = tables
    fk1 = FineKick(L, pm3_mode=CUBE_PM3_PERIODIC, apm3f=Ln.SHORT.apm3f)
    a1 = apm3_table(Ln.SHORT.apm3f)
    rho, idx, xp, vp = Ln.device_image(img, dev)
    vp0 = vp.clone()
    out = torch.zeros(8, device=dev)
    a_mid, dt = float(np.float32(6 * np.pi)), 1.0

    def kick(with_shell=True):
        fk1.kick_fine_device(rho, idx, xp, img.n_used, vp, out, isort, ires, ix, a1, rs, 1.0, a_mid, dt, stream=stream)
        if with_shell:
            shell.kick(rho, idx, xp, img.n_used, vp, scale, a_mid, dt, stream=stream)
    for _ in range(max(args.warmup, 0)):
        kick()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        kick()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    res = {"ms_per_step": ms, "value": img.n_particles / (ms * 1e-3), "unit": UNIT,
           "speedup_vs_plain": ms_plain / ms, "pp_cutoff_fine_cells": Ln.SHORT.cutoff,
           "train": tinfo}
    # errors against the FP64 truth on the plain run's sampled particles
    if truth_plain is not None and not args.no_truth:
        act = np.nonzero(img.active)[0]
        rng = np.random.default_rng(12345)
        samp = rng.choice(act, min(args.truth_targets, act.size), replace=False)
        Ft = force_truth_fp64(W.physical_positions(img), float(L.ng), L.app, img.pid[samp])
        kc = Ln.kick_coef(a_mid, dt)

        def err(with_shell):
            vp.copy_(vp0)
            kick(with_shell)
            torch.cuda.synchronize()
            F = (vp - vp0).cpu().numpy().reshape(-1, 3).astype(np.float64)[samp] / kc
            d = np.linalg.norm(F - Ft, axis=1)
            m = np.linalg.norm(Ft, axis=1)
            return float(np.sqrt(np.sum(d ** 2) / np.sum(m ** 2))), float(np.percentile(d / np.maximum(m, 1e-30), 99))
        rms, p99 = err(True)
        rms0, p990 = err(False)
        res["force_error"] = {"rms_rel": rms, "p99_rel": p99, "targets": int(samp.size)}
        res["force_error_cutoff1_without_shell"] = {"rms_rel": rms0, "p99_rel": p990}
        res["bound"] = LEARNED_BOUND
        res["fallback"] = bool(rms > LEARNED_BOUND)
        res["note"] = ("the sampled error exceeds the bound: the kick falls back to the plain cutoff-2 kick, "
                       "whose value is the line's value" if rms > LEARNED_BOUND else
                       "within the bound: the learned kick stands")
        # the per-cell check: the network against the full-cutoff kick cell by cell, and the cells
        # over the bound take its velocities (cube_learned_fallback)
        try:
            res["per_cell_fallback"] = per_cell_fallback(args, img, tables, stream, kick, vp, vp0, Ft, samp, kc,
                                                         ms_plain)
        except Exception as e:  # reported beside the learned kick, never instead of it
            res["per_cell_fallback"] = {"error": repr(e)}
    shell.close()
    return res


FALLBACK_SAMPLES = 4  # particles checked per coarse cell


def per_cell_fallback(args, img, tables, stream, learned_kick, vp, vp0, Ft, samp, kc, ms_plain):
    """The learned kick with its per-cell check: learned kick, full-cutoff kick on a copy of the
    starting velocities, then every coarse cell checked on its first FALLBACK_SAMPLES particles
    against the full-cutoff kick and the cells over the bound recomputed at cutoff 2 (they take
    the full-cutoff velocities).  Timed over the same steps as the plain kick; the error after
    the fallback is stated against the FP64 truth on the same sampled particles."""
    import torch
    from cube2_b200 import learned as Ln
    from cube2_b200.kick import CUBE_PM3_PERIODIC, FineKick
    from cube2_b200.layout import apm3_table
    L = img.layout
    isort, ires, ix, _, rs = tables
    rho, idx, xp, _ = Ln.device_image(img, vp.device)
    fk1 = FineKick(L, pm3_mode=CUBE_PM3_PERIODIC, apm3f=Ln.SHORT.apm3f)
    fk2 = FineKick(L, pm3_mode=CUBE_PM3_PERIODIC, apm3f=Ln.PLAIN.apm3f)
    a2 = apm3_table(Ln.PLAIN.apm3f)
    vpf = vp0.clone()
    out = torch.zeros(8, device=vp.device)
    a_mid, dt = float(np.float32(6 * np.pi)), 1.0

    def step():  # the layout's PM3 softening is switched between the two splits (cube_set_layout)
        vp.copy_(vp0)
        fk1.configure()
        learned_kick(True)
        vpf.copy_(vp0)
        fk2.configure()
        fk2.kick_fine_device(rho, idx, xp, img.n_used, vpf, out, isort, ires, ix, a2, rs, 1.0, a_mid, dt,
                             stream=stream)
        return Ln.fallback(rho, idx, img.n_used, vp0, vp, vpf, LEARNED_BOUND, FALLBACK_SAMPLES, stream=stream)
    for _ in range(max(args.warmup, 1)):
        st = step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        st = step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    F = (vp - vp0).cpu().numpy().reshape(-1, 3).astype(np.float64)[samp] / kc
    d = np.linalg.norm(F - Ft, axis=1)
    m = np.linalg.norm(Ft, axis=1)
    return {"bound": LEARNED_BOUND, "samples_per_cell": FALLBACK_SAMPLES, **st,
            "fraction_fallen_back": st["particles_fallen_back"] / max(img.n_particles, 1),
            "force_error_after": {"rms_rel": float(np.sqrt(np.sum(d ** 2) / np.sum(m ** 2))),
                                  "p99_rel": float(np.percentile(d / np.maximum(m, 1e-30), 99))},
            "ms_per_step": ms, "value": img.n_particles / (ms * 1e-3), "unit": UNIT,
            "speedup_vs_plain": ms_plain / ms,
            "what": "learned kick + full-cutoff kick (the reference for the check) + per-cell check and fallback, per step"}


def _batch_boxes(workload: str):
    from cube2_b200 import ic
    from cube2_b200 import workloads as W
    w = W.WORKLOADS[workload]
    return [ic.zeldovich_box(int(m), float(w["box"]), 0.5, w["seed"] + t) for t, m in enumerate(W.batch_counts(workload))]


def batch_truth(workload: str, img, samp, force_truth_fp64):
    """FP64 truth for the sampled stored particles of a batch: each box is summed alone."""
    from cube2_b200 import workloads as W
    from cube2_b200.layout import build_image
    tl = W.tile_layout(workload)
    boxes = _batch_boxes(workload)
    n_per = np.array([b[0].shape[0] for b in boxes])
    poffs = np.concatenate([[0], np.cumsum(n_per)])
    pid = img.pid[samp]
    box = np.searchsorted(poffs, pid, side="right") - 1
    F = np.zeros((samp.size, 3))
    for t in np.unique(box):
        sel = np.nonzero(box == t)[0]
        one = build_image(boxes[t][0], boxes[t][1], tl)
        pos = W.physical_positions(one)
        F[sel] = force_truth_fp64(pos, float(tl.ng), tl.app, pid[sel] - poffs[t])
    return F


def batch_leg(workload: str, stream, steps: int, warmup: int):
    """Batched uneven boxes beside the main kick: every box of the batch workload in one kick
    (one periodic mesh per box, one batched transform, one persistent PP launch over all boxes),
    timed with CUDA events over K steps after W warm-up steps (the first one autotunes the PP
    shape), then replayed as a captured CUDA graph, then against one kick call per box."""
    import torch
    from cube2_b200 import workloads as W
    from cube2_b200.kick import CUBE_PM3_TILE_PERIODIC, FineKick
    w = W.WORKLOADS[workload]
    img = W.make(workload)
    L = img.layout
    isort, ires, ix, apm3, rs = W.tables(workload)
    fk = FineKick(L, pm3_mode=CUBE_PM3_TILE_PERIODIC, apm3f=w["apm3f"])
    dev = torch.device("cuda", torch.cuda.current_device())
    d_rhoc = torch.from_numpy(img.rhoc.reshape(-1).copy()).to(dev)
    d_idx = torch.from_numpy(img.idx_b_r.reshape(-1).copy()).to(dev)
    d_xp = torch.from_numpy(img.xp.reshape(-1).copy()).to(dev)
    d_vp = torch.from_numpy(img.vp.reshape(-1).copy()).to(dev)
    d_out = torch.zeros(8, dtype=torch.float32, device=dev)
    a_mid, dt = np.float32(6 * np.pi), np.float32(1.0)

    def kick():
        fk.kick_fine_device(d_rhoc, d_idx, d_xp, img.n_used, d_vp, d_out, isort, ires, ix, apm3, rs, 1.0, a_mid,
                            dt, stream=stream)
    for _ in range(max(warmup, 1)):
        kick()
    torch.cuda.synchronize()
    err_word = int(d_out[5:6].cpu().view(torch.int32).item())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        kick()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(steps, 1)
    gms = None
    kg = fk.kick_graph(d_rhoc, d_idx, d_xp, img.n_used, d_vp, d_out, isort, ires, ix, apm3, rs, 1.0, a_mid, dt)
    try:
        for _ in range(max(warmup, 1)):
            kg.launch(stream)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            kg.launch(stream)
        e1.record(stream)
        torch.cuda.synchronize()
        gms = e0.elapsed_time(e1) / max(steps, 1)
    finally:
        kg.close()
    from cube2_b200.kick import pp_shapes
    table, cur = pp_shapes()
    loop = per_box_loop(workload, fk, img, stream, a_mid, dt, ms)
    n_per = np.array([b ** 3 for b in W.batch_counts(workload)])
    return {"workload": workload, "boxes": int(L.nnt ** 3), "box_fine_cells": w["box"],
            "particles": int(img.n_particles), "stored": int(img.n_used),
            "particles_per_box": {"min": int(n_per.min()), "median": int(np.median(n_per)), "max": int(n_per.max())},
            "ms_per_step": ms, "value": img.n_particles / (ms * 1e-3), "unit": UNIT,
            "graph_ms_per_step": gms, "graph_value": img.n_particles / (gms * 1e-3) if gms else None,
            "per_box_loop": loop, "batched_speedup_vs_per_box_loop": loop["ms_per_step"] / ms,
            "pp_shape": {k: table[cur][k] for k in ("chunk", "jtile", "unroll", "blocks", "packed")},
            "device_error_mask": err_word,
            "what": "all boxes in one kick (CUBE_PM3_TILE_PERIODIC: one 64^3 periodic mesh per box, one batched "
                    "transform, one persistent PP launch over every box's work items), plain launches and as a "
                    "replayed CUDA graph, against one cube_kick_fine_device call per box"}


def per_box_loop(workload: str, fk_batch, img, stream, a_mid, dt, ms_batched):
    """The same boxes kicked one call per box (device-resident, one-tile layout), timed with
    CUDA events over one pass after a warm-up pass: the launch-per-tile loop the batch replaces."""
    import torch
    from cube2_b200 import workloads as W
    from cube2_b200.kick import CUBE_PM3_PERIODIC, FineKick
    from cube2_b200.layout import RATIO_SF, apm3_table, build_image, ixyz3_table
    w = W.WORKLOADS[workload]
    tl = W.tile_layout(workload)
    dev = torch.device("cuda", torch.cuda.current_device())
    ones = [build_image(p, v, tl) for p, v in _batch_boxes(workload)]

    def up(a):
        return torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).to(dev)
    bufs = [(up(o.rhoc), up(o.idx_b_r), up(o.xp), up(o.vp), o.n_used) for o in ones]
    d_out = torch.zeros(8, dtype=torch.float32, device=dev)
    fk1 = FineKick(tl, pm3_mode=CUBE_PM3_PERIODIC, apm3f=w["apm3f"])
    t1 = (np.arange(1, tl.ns3 + 1, dtype=np.int32), np.full(tl.ns3, 2, np.int32), ixyz3_table(tl),
          apm3_table(w["apm3f"]), RATIO_SF.copy())

    def one_pass():
        for b in bufs:
            fk1.kick_fine_device(b[0], b[1], b[2], b[4], b[3], d_out, *t1, 1.0, a_mid, dt, stream=stream)
    one_pass()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    one_pass()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return {"ms_per_step": ms, "value": img.n_particles / (ms * 1e-3), "unit": UNIT, "calls_per_step": len(bufs),
            "batched_speedup": ms / ms_batched,
            "what": "one cube_kick_fine_device call per box (one-tile layout, periodic mesh per call)"}


# ------------------------------------------------------------------------------------------------
# reference CPU path (the baseline leg and the reference arm)


def _nnest_for_host():
    n = os.cpu_count() or 1
    best = 8
    for k in (8, 16, 32, 64, 128, 256):
        if k <= n:
            best = k
    return best


def reference_setup(workload: str, img):
    """The reference CPU path for the workload's image: the reference's own PP kernel
    (pp_force_kernel.c, compiled for this layout and nnest host threads) and the PM3 Green
    table, tabulated in FP64 on the host by the restatement of Green.f90 (outside any timed
    region).  Nothing of this library is loaded."""
    from cube2_b200 import workloads as W
    from oracle import oracle as O
    w = W.WORKLOADS[workload]
    L = img.layout
    nnest = _nnest_for_host()
    ref = O.RefPP(L, nnest=nnest)
    n = L.ng * w["rsf"]
    t = time.perf_counter()
    G = O.green_mirrored(n, w["apm3f"], 0.0, 1.0 / w["rsf"])
    return {"ref": ref, "G": G, "nnest": nnest, "green_seconds": time.perf_counter() - t, "mesh": n}


def reference_step(workload: str, img, setup):
    """One fine-scale kick of the whole image through the reference CPU path: the reference's
    c_pp_force_kernel over every parent tile (pp_force_kernel.c:393-445) and the PM3
    restatement of kick.f90 pm_thread on the full periodic mesh (float32 FFT standing in for
    sfftw).  Returns (seconds of PP, seconds of PM3)."""
    from cube2_b200 import workloads as W
    from oracle import oracle as O
    w = W.WORKLOADS[workload]
    L = img.layout
    isort, ires, ix, apm3, rs = W.tables(workload)
    a_mid, dt = np.float32(6 * np.pi), np.float32(1.0)
    t = time.perf_counter()
    setup["ref"].kick(img, [int(ires[0])] * L.nnt ** 3, apm3, rs, 1.0, a_mid, dt)
    t_pp = time.perf_counter() - t
    t = time.perf_counter()
    O.pm3_periodic(img, w["rsf"], setup["G"], 1.0, a_mid, dt, fft_dtype=np.float32)
    return t_pp, time.perf_counter() - t


def _reference_sample(img, setup) -> str:
    L = img.layout
    return (f"the whole image every step: pp_force_kernel.c c_pp_force_kernel over all {L.nnt ** 3} parent tiles "
            f"({setup['nnest']} OpenMP threads) + the PM3 restatement of kick.f90 pm_thread on the full "
            f"{setup['mesh']}^3 periodic mesh (scipy pocketfft float32 standing in for sfftw); Green table "
            f"tabulated on the host in FP64 beforehand ({setup['green_seconds']:.1f} s, untimed)")


def cpu_reference(workload: str, img):
    """The cpu_baseline leg: one kick of the whole image through the reference CPU path."""
    setup = reference_setup(workload, img)
    t_pp, t_pm3 = reference_step(workload, img, setup)
    return {"value": img.n_particles / (t_pp + t_pm3), "unit": UNIT, "cores": int(setup["nnest"]),
            "kind": "reference", "pm3_kind": "port", "seconds_pp": t_pp, "seconds_pm3": t_pm3,
            "host_cores": int(os.cpu_count() or 1), "sample": _reference_sample(img, setup)}


LOOP_METRIC = "particle-steps/s (drift + kick + buffer_v)"
LOOP_UNIT = "particle-steps/s"


def _timed_steps(loop, steps, stream):
    """K steps of a TimeLoop timed with CUDA events on its stream; (ms per step, drift ms, kick ms)."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for k in range(steps):
        loop.step(events=ev[k])
    torch.cuda.synchronize()
    drift = sum(e[0].elapsed_time(e[1]) for e in ev)
    kick = sum(e[1].elapsed_time(e[2]) for e in ev)
    return ev[0][0].elapsed_time(ev[-1][2]) / max(steps, 1), drift / max(steps, 1), kick / max(steps, 1)


def loop_leg(workload: str, steps: int, warmup: int, dev, stream, variant_names=("learned", "learned_lognormal_boxes",
                                                                            "cutoff1_without_shell"), world: int = 1):
    """The kick-drift time loop (drift, buffer_grid, buffer_x, kick, buffer_v per step) on
    Zel'dovich initial conditions built on the device.  The plain loop (cutoff 2) is timed;
    the same start is then run with the learned shell (cutoff 1 + MLP) and with cutoff 1 alone,
    and the final states are compared with the plain one by CIC power-spectrum ratio (k up to
    k_Nyquist / 2 of the P(k) grid) and rms position difference."""
    import torch
    from cube2_b200 import learned as Ln
    from cube2_b200 import loop as LP
    from cube2_b200 import workloads as W
    from cube2_b200.layout import Layout
    w = W.LOOP_WORKLOADS[workload]
    L = Layout(**w["layout"])
    t0 = time.perf_counter()
    di, dt, c = LP.start_with_growth(L, w["rms"], w["seed"], w["growth_per_step"], w["apm3f"], dev)
    torch.cuda.synchronize()
    t_ic = time.perf_counter() - t0
    N = L.ng ** 3
    nw = w["pk_grid"]
    pk0 = di.power_spectrum(nw)
    start_learned, start_short = LP.clone_image(di), LP.clone_image(di)
    plain = LP.TimeLoop(di, w["apm3f"], coef=dt, dt_mid=dt, stream=stream)
    for _ in range(max(warmup, 0)):
        plain.step()
    torch.cuda.synchronize()
    if plain.error_word():
        raise RuntimeError(f"device error mask {plain.error_word()}")
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    clocks = Clocks(uuid)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    ms, ms_drift, ms_kick = _timed_steps(plain, steps, stream)
    ck = clocks.stop()
    ms = max_over_ranks(ms, world, dev)
    pk_plain = di.power_spectrum(nw)
    n_phys_ok = di.n_physical == N

    def run_variant(start, apm3f, shell=None, scale=1.0):
        lp = LP.TimeLoop(start, apm3f, coef=dt, dt_mid=dt, shell=shell, shell_scale=scale, stream=stream)
        for _ in range(max(warmup, 0)):
            lp.step()
        m, md, mk = _timed_steps(lp, steps, stream)
        pk = start.power_spectrum(nw)
        kmax = nw // 4
        ok = (pk_plain["modes"] > 0) & (np.arange(pk_plain["modes"].size) >= 1) & (np.arange(pk_plain["modes"].size) <= kmax)
        ratio = pk["pk"][ok] / pk_plain["pk"][ok]
        return {"ms_per_step": m, "drift_ms": md, "kick_ms": mk, "value": N / (m * 1e-3), "unit": LOOP_UNIT,
                "pk_ratio_max_dev": float(np.max(np.abs(ratio - 1.0))),
                "pk_ratio_bins": [round(float(x), 5) for x in ratio],
                "rms_position_difference_fine_cells": LP.rms_position_difference(start, di),
                "within_1pct": bool(np.max(np.abs(ratio - 1.0)) <= 0.01), "error_word": lp.error_word()}
    variants = {}
    start_lognormal = LP.clone_image(start_learned) if "learned_lognormal_boxes" in variant_names else None
    if "learned" in variant_names:
        try:
            # the method's own snapshots: a 128^3 companion box of the same statistics (another seed),
            # every 5 steps of a plain loop as long as this one
            sl = dict(w["layout"], ng=128)
            snaps = LP.snapshots(Layout(**sl), w["rms"], w["seed"] + 7, w["growth_per_step"], w["apm3f"],
                                 warmup + steps, 2, dev)
            shell, scale, tinfo = Ln.train_shell_on(snaps, dev, steps=12000,
                                                    fields="snapshots 0, 2, 4, ... of a plain 128^3 loop of the "
                                                    f"same statistics (seed {w['seed'] + 7})")
            del snaps
            variants["learned"] = run_variant(start_learned, 2.0, shell, scale)
            variants["learned"]["train"] = tinfo
            shell.close()
        except Exception as e:  # reported beside the plain loop, never instead of it
            variants["learned"] = {"error": repr(e)}
    if start_lognormal is not None:
        try:
            shell, scale, tinfo = Ln.train_shell(dev)
            variants["learned_lognormal_boxes"] = run_variant(start_lognormal, 2.0, shell, scale)
            variants["learned_lognormal_boxes"]["train"] = tinfo
            shell.close()
        except Exception as e:
            variants["learned_lognormal_boxes"] = {"error": repr(e)}
    if "cutoff1_without_shell" in variant_names:
        try:
            variants["cutoff1_without_shell"] = run_variant(start_short, 2.0)
        except Exception as e:
            variants["cutoff1_without_shell"] = {"error": repr(e)}
    growth = pk_plain["pk"][1:nw // 4 + 1] / pk0["pk"][1:nw // 4 + 1]
    return {"workload": workload, "particles": N, "layout": L.as_dict(), "pm3_mesh": L.ng * 2,
            "pp_cutoff_fine_cells": w["apm3f"] / 2, "growth_per_step": w["growth_per_step"], "dt": dt,
            "growth_rate_c": c, "steps": steps, "warmup": warmup, "ms_per_step": ms, "value": N * world / (ms * 1e-3),
            "unit": LOOP_UNIT, "stages_ms": {"drift_and_buffers": ms_drift, "kick_and_buffer_v": ms_kick},
            "initial_conditions_seconds": t_ic, "particles_conserved": bool(n_phys_ok),
            "pk_growth_plain": [round(float(x), 4) for x in growth[:8]], "pk_grid": nw, "variants": variants,
            "clocks": ck}


def run_loop(args, rank, world, local_rank):
    """--workload loop*: the time loop as the bench line itself (see loop_leg)."""
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world > 1:
        dist.init_process_group("nccl", device_id=dev)
    stream = torch.cuda.Stream(dev)
    names = () if (rank != 0 or args.no_learned) else ("learned", "learned_lognormal_boxes", "cutoff1_without_shell")
    r = loop_leg(args.workload, args.steps, args.warmup, dev, stream, names, world)
    peak, src = measured_hbm_peak()
    line = {"metric": LOOP_METRIC, "value": r["value"], "unit": LOOP_UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32 (int16 fixed-point positions, fp64 Green table)",
            "data": "synthetic (Zel'dovich lattice, P(k) ~ k^-2, built on the device; see cube2_b200/loop.py)",
            "config": {"workload": args.workload, "particles": r["particles"], "layout": r["layout"],
                       "pm3_mesh": r["pm3_mesh"], "pp_cutoff_fine_cells": r["pp_cutoff_fine_cells"],
                       "growth_per_step": r["growth_per_step"], "dt": r["dt"], "growth_rate_c": r["growth_rate_c"],
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (mesh 1024^3 fp32 = 4.3 GB, particle arrays > 3 GB)"},
            "stages_ms": r["stages_ms"], "initial_conditions_seconds": r["initial_conditions_seconds"],
            "particles_conserved": r["particles_conserved"], "pk_growth_plain": r["pk_growth_plain"],
            "pk_grid": r["pk_grid"], "variants": r["variants"], "clocks": r["clocks"], "hbm_peak_gbs": peak,
            "e2e": {"unavailable": "the loop keeps the image on the device between steps; the host-array "
                                   "entry points (cube_kick_fine, cube_drift) are timed on the single-kick workloads"},
            "cpu_baseline": {"unavailable": "the reference loop is the Fortran driver (no Fortran compiler here)"}}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def run_reference(args, rank, world):
    """The reference arm: the reference's own CPU implementation of the path on the host
    cores, every step a full kick of the whole image (warm-up steps untimed)."""
    if rank != 0:
        return
    from cube2_b200 import workloads as W
    if args.workload in W.LOOP_WORKLOADS:
        print(json.dumps({"impl": "reference", "unavailable": "the reference's time loop is the Fortran driver "
                          "(main.f90); no Fortran compiler here"}))
        return
    if W.WORKLOADS[args.workload]["kind"] == "batch":
        print(json.dumps({"impl": "reference", "unavailable": "the reference CPU path is timed on the single-image "
                          "workloads; batch workloads compare against a per-box launch loop instead"}))
        return
    img = W.make(args.workload)
    setup = reference_setup(args.workload, img)
    pp, pm3 = [], []
    for s in range(args.warmup + args.steps):
        t_pp, t_pm3 = reference_step(args.workload, img, setup)
        if s >= args.warmup:
            pp.append(t_pp)
            pm3.append(t_pm3)
    sec = float(np.mean(np.array(pp) + np.array(pm3))) if pp else float("nan")
    value = img.n_particles / sec
    w = W.WORKLOADS[args.workload]
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
            "config": {"workload": args.workload, "particles": img.n_particles, "pm3_mesh": img.layout.ng * w["rsf"],
                       "pp_cutoff_fine_cells": w["apm3f"] / w["rsf"], "softening_fine_cells": img.layout.app},
            "stages_ms": {"pp": 1e3 * float(np.mean(pp)), "pm3": 1e3 * float(np.mean(pm3))},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": int(setup["nnest"]), "kind": "reference",
                             "pm3_kind": "port", "host_cores": int(os.cpu_count() or 1),
                             "sample": _reference_sample(img, setup)},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    rank, world, local_rank = dist_env()
    from cube2_b200 import workloads as W
    if args.impl == "reference":
        run_reference(args, rank, world)
    elif args.workload in W.LOOP_WORKLOADS:
        run_loop(args, rank, world, local_rank)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
