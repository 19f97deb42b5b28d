"""Benchmark of the KerrTrace hot path on B200.

One step = one 1920x1080 frame of the c2 scene (a = 0.998, r_obs 100 M, inclination 85 deg,
tolerance 1e-6, up to 20000 DP5(4) steps per ray, FBM-modulated Novikov-Thorne disk, bloom
radius 24, ACES + sRGB): the trace kernel plus the post-processing kernel.

  value   Mrays/s over all ranks, device-timed (CUDA events around each step on the launch
          stream; L2 flushed between steps by writing a 256 MiB buffer outside the timed events)
  e2e     the same metric through the public renderer API (kt_renderer_submit_render +
          ready_frame + finish_frame): per frame the camera goes host -> device as launch
          arguments and the 0x00RRGGBB frame plus its LUT error word come back into pinned
          host memory; two frames in flight as the reference host keeps them (the copy of one
          overlaps the trace of the next); wall-clock from the first submit to the last frame
          handed back
  roofline  FP32 work of the trace kernel (counted RHS evaluations / attempts / steps x the
          static op counts in kerrtrace_b200/flops.py) / its event-timed duration, against the
          FP32 FMA throughput measured on the same GPU before the timed region (kt_fma_peak)
  cpu_baseline  the CPU oracle (f64 restatement, all host cores) on a strided sample of the
          same frame

--impl reference runs the reference's own cuda/kernel.cu (compiled from source into
oracle/_ref) with the launch sequence of src/renderer/mod.rs: trace_kernel, bloom_horizontal,
post_process, image copy to pinned host memory.

Multi-GPU (torchrun): every rank renders its own frame of the same scene seen from a different
azimuth (the spacetime is axisymmetric, so every rank has the same work): weak scaling, no
data-path collective; the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))


# DRAM bytes per ray of the trace kernel from an ncu capture of the c2 scene at 960x540
# (dram__bytes_read.sum 149504 B + dram__bytes_write.sum 0 B over 518400 rays): the HDR output
# stays in L2, the kernel reads only its LUTs and parameters.
TRACE_TRAFFIC_PER_RAY = 149504 / 518400


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2")
    ap.add_argument("--schedule", default="auto", choices=["auto", "wavefront", "plain"])
    ap.add_argument("--mode", default="ref", choices=["ref", "spec"],
                    help="semantics of the main loop: the reference's (default) or stated physics")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "mixed", "fp64"],
                    help="arithmetic of the main loop (mixed / fp64 need --mode spec)")
    ap.add_argument("--no-precision", action="store_true")
    ap.add_argument("--no-retirement", action="store_true",
                    help="skip the leg that times the frame with NaN-frozen rays kept to max_steps")
    ap.add_argument("--no-c3", action="store_true", help="skip the 4096^2 x 8-draw precision ablation")
    ap.add_argument("--no-sequence", action="store_true", help="skip the headless frame-sequence leg")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--batch-scale", type=int, default=1,
                    help="divide the batched workload's frame sizes by this (small cases for profiling)")
    ap.add_argument("--no-pareto", action="store_true",
                    help="skip the accuracy-against-speed sweep of FP32 / mixed / FP64 over tolerances")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--size", default=None, help="WxH override of the scene resolution (same scene otherwise)")
    ap.add_argument("--tuning", default=None,
                    help="schedule,block_x,block_y,blocks_per_sm,refill_min,order: this launch shape instead of "
                         "the autotuner's (reproducible profiling)")
    return ap.parse_args()


class ClockSampler:
    """NVML sampling (every 5 ms, in a thread) of the SM clock and the clock-event reasons
    during the timed region."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown"}

    def __init__(self, device_index: int, period_s: float = 0.005):
        self.dev = device_index
        self.period = period_s
        self.samples = []
        self._stop = None
        self._thread = None
        self.max_mhz = None

    def __enter__(self):
        import threading
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.dev)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
        except Exception:  # no NVML: the summary says so
            return self
        self._stop = threading.Event()

        def run():
            while not self._stop.is_set():
                try:
                    mhz = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                    why = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    pw = pynvml.nvmlDeviceGetPowerUsage(h) / 1000.0
                    self.samples.append((float(mhz), int(why), pw))
                except Exception:
                    pass
                self._stop.wait(self.period)

        self._thread = threading.Thread(target=run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *exc):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=2)

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"]}
        sm = sorted(x[0] for x in self.samples)
        reasons = sorted({name for _, why, _ in self.samples for bit, name in self.REASONS.items() if why & bit})
        return {"sm_mhz": sm[len(sm) // 2], "sm_mhz_min": sm[0], "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "power_w_max": round(max(x[2] for x in self.samples), 1), "samples": len(self.samples)}


def dist_setup(backend: str = "nccl"):
    """One process per GPU (RANK / LOCAL_RANK / WORLD_SIZE / MASTER_* from torchrun).  The
    process group only carries the barrier and the max-over-ranks time; `gloo` runs the same
    host logic on CPU (tests)."""
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if backend == "nccl":
        torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        kw = {"device_id": torch.device("cuda", local)} if backend == "nccl" else {}
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300), **kw)
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_mrays_s(rays_per_rank: int, world: int, max_ms: float) -> float:
    """Whole-job throughput: the rays of all ranks over the slowest rank's time (weak scaling:
    every rank traces its own frame of the same size)."""
    return rays_per_rank * world / (max_ms / 1e3) / 1e6


def rank_camera(workloads, name, rank, world, size=None, host=None):
    """The scene of this rank: the named workload (optionally at another resolution) seen from
    azimuth 360 * rank / world.  `host` supplies the scene's host arithmetic (the library's, or
    the oracle's restatement in the reference arm)."""
    cfg, cam = workloads.scene(name, host=host)
    if size:
        w, h = (int(v) for v in size.lower().split("x"))
        cfg = workloads.scaled(cfg, w, h)
    if world > 1 and rank > 0:
        r = math.sqrt(sum(c * c for c in cam.cam_pos))
        incl = math.degrees(math.acos(cam.cam_pos[1] / r))
        fov = 2 * math.degrees(math.atan(cam.fov_scale))
        cam = workloads.orbit_camera(r, incl, fov, azimuth_deg=360.0 * rank / world, host=host)
    return cfg, cam


def workload_label(name: str, cfg) -> str:
    """config.workload of both arms: the scene and the values that size its work."""
    return (f"{name}: {cfg.width}x{cfg.height}, a={cfg.spin:.3f}, tol={cfg.tolerance:g}, "
            f"max_steps={cfg.max_steps}, spp={cfg.spp}, bloom r={cfg.bloom_radius:g}")


def cpu_baseline(cfg, cam, budget_s: float) -> dict:
    """The CPU oracle (f64, reference semantics, all host cores): whole frames of the same scene
    until `budget_s` has elapsed, or a strided pixel sample when one frame would exceed it."""
    import numpy as np

    import oracle
    threads = os.cpu_count() or 1
    sc = oracle.Scene(cfg, cam, tex_mode=1)
    n = cfg.width * cfg.height
    probe = np.arange(0, n, 64, dtype=np.int64)
    t0 = time.perf_counter()
    sc.render(2, pixels=probe, threads=threads)
    est_frame = (time.perf_counter() - t0) * 64
    if est_frame <= budget_s:
        frames, t = 0, 0.0
        while t < budget_s and frames < 20:
            t0 = time.perf_counter()
            sc.render(2, threads=threads)
            t += time.perf_counter() - t0
            frames += 1
        rays = frames * n * cfg.spp
        sample = f"f64 oracle, {frames} whole {cfg.width}x{cfg.height} frame(s) in {t:.2f} s"
    else:
        stride = max(1, int(math.ceil(est_frame / budget_s)))
        pix = np.arange(0, n, stride, dtype=np.int64)
        t0 = time.perf_counter()
        sc.render(2, pixels=pix, threads=threads)
        t = time.perf_counter() - t0
        rays = len(pix) * cfg.spp
        sample = f"f64 oracle, every {stride}th pixel of the {cfg.width}x{cfg.height} frame ({len(pix)} pixels) in {t:.2f} s"
    return {"value": round(rays / t / 1e6, 4), "unit": "Mrays/s", "cores": threads, "kind": "port", "sample": sample}


def retirement_leg(ctx, cfg, cam, stream, reps: int = 2) -> dict:
    """The same frame with retirement of NaN-frozen rays switched off (tuning keep_frozen = 1):
    frozen rays then iterate to max_steps as the reference's do (cuda/kerr_trace.cuh:62,83-125),
    so the trace does the reference's amount of work with this library's kernel.  Event-timed
    trace of both settings on the tuned launch shape and on the default persistent shape (the
    faster of the two is reported), the bit-identity of the two images and the work counters."""
    import torch

    import kerrtrace_b200 as kt
    n = cfg.width * cfg.height
    a = torch.zeros((n, 4), device="cuda")
    b = torch.zeros((n, 4), device="cuda")
    err = torch.zeros(2, dtype=torch.int32, device="cuda")
    tuned = ctx.tuning().as_dict()
    shapes = {"tuned": tuned, "wavefront_default": dict(schedule=kt.SCHED_WAVEFRONT, block_x=0, block_y=0,
                                                        blocks_per_sm=4, refill_min=1, order=0)}

    def timed(out, k):
        ctx.trace(cam, out.data_ptr(), err.data_ptr(), stream, kt.SCHED_AUTO)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(k):
            ctx.trace(cam, out.data_ptr(), err.data_ptr(), stream, kt.SCHED_AUTO)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k

    res = {}
    for label, shape in shapes.items():
        shape = {k: v for k, v in shape.items() if k != "keep_frozen"}
        ctx.set_tuning(**shape, keep_frozen=0)
        t_retire = timed(a, max(3, reps))
        ctx.set_tuning(**shape, keep_frozen=1)
        t_keep = timed(b, reps)
        res[label] = {"retire_ms": round(t_retire, 4), "keep_frozen_ms": round(t_keep, 4),
                      "bit_identical": bool(torch.equal(a.view(torch.int32), b.view(torch.int32)))}
    ctx.set_tuning(**{k: v for k, v in tuned.items() if k != "keep_frozen"}, keep_frozen=1)
    st_keep = ctx.trace_counted(cam, b.data_ptr(), err.data_ptr(), stream, kt.SCHED_AUTO)
    ctx.set_tuning(**tuned)
    st = ctx.trace_counted(cam, a.data_ptr(), err.data_ptr(), stream, kt.SCHED_AUTO)
    best = min(res, key=lambda k: res[k]["keep_frozen_ms"])
    out = {"shapes": res, "keep_frozen_best": best,
           "keep_frozen_trace_ms": res[best]["keep_frozen_ms"], "retire_trace_ms": res["tuned"]["retire_ms"],
           "retirement_gain": round(res[best]["keep_frozen_ms"] / res["tuned"]["retire_ms"], 2),
           "keep_frozen_mrays_s": round(n * cfg.spp / res[best]["keep_frozen_ms"] / 1e3, 3),
           "bit_identical": all(r["bit_identical"] for r in res.values()),
           "frozen_rays": int(st.frozen_rays),
           "work_retire": {"steps": int(st.steps), "attempts": int(st.attempts), "rhs_evals": int(st.rhs_evals)},
           "work_keep_frozen": {"steps": int(st_keep.steps), "attempts": int(st_keep.attempts),
                                "rhs_evals": int(st_keep.rhs_evals)}}
    return out


def precision_leg(cfg, cam, local, reps: int) -> dict:
    """Stated-physics traces of the same frame in FP32, mixed precision and FP64: Mrays/s of
    each (trace kernel, event-timed, autotuned launch shape) and the per-pixel error of FP32 and
    mixed against the FP64 run (HDR RGB, and radius / redshift of the first disk hit)."""
    import numpy as np
    import torch

    import kerrtrace_b200 as kt
    from kerrtrace_b200 import autotune

    n = cfg.width * cfg.height
    hdr = torch.zeros((n, 4), device="cuda")
    aux = torch.zeros((n, 4), device="cuda")
    err = torch.zeros(2, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    out, runs = {}, {}
    for name, prec in (("fp64", kt.PREC_FP64), ("fp32", kt.PREC_FP32), ("mixed", kt.PREC_MIXED)):
        c = cfg.copy()
        c.mode, c.precision = kt.MODE_SPEC, prec
        ctx = kt.Context(c, local)
        tuned = autotune.autotune(ctx, cam, reps=2, stream=stream)
        st = ctx.trace_counted(cam, hdr.data_ptr(), err.data_ptr(), stream, kt.SCHED_AUTO, aux.data_ptr())
        out[name] = (hdr.cpu().numpy()[:, :3].astype(np.float64), aux.cpu().numpy().astype(np.float64))
        ctx.trace(cam, hdr.data_ptr(), err.data_ptr(), stream, kt.SCHED_AUTO)
        torch.cuda.synchronize()
        k = max(1, reps if prec != kt.PREC_FP64 else reps // 3)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(k):
            ctx.trace(cam, hdr.data_ptr(), err.data_ptr(), stream, kt.SCHED_AUTO)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / k
        runs[name] = {"mrays_s": round(n * cfg.spp / ms / 1e3, 2), "trace_ms": round(ms, 4), "steps": int(st.steps),
                      "fp64_zone_steps": int(st.fp64_steps), "tuning": tuned.best}
        ctx.close()
    ref, ref_aux = out["fp64"]
    floor = 1e-6 * np.abs(ref).max()
    for name in ("fp32", "mixed"):
        a, a_aux = out[name]
        rel = (np.abs(a - ref) / np.maximum(np.abs(ref), floor)).max(1)
        hit = np.isfinite(a_aux[:, 0]) & np.isfinite(ref_aux[:, 0])
        rr = np.abs(a_aux[hit, 0] - ref_aux[hit, 0]) / np.abs(ref_aux[hit, 0])
        rg = np.abs(a_aux[hit, 1] - ref_aux[hit, 1]) / np.abs(ref_aux[hit, 1])
        runs[name]["err_vs_fp64"] = {
            "hdr_p99": float(np.quantile(rel, 0.99)), "hdr_p999": float(np.quantile(rel, 0.999)),
            "hdr_frac_over_1e-3": float(np.mean(rel > 1e-3)),
            "r_cross_p99": float(np.quantile(rr, 0.99)) if hit.any() else None,
            "g_p99": float(np.quantile(rg, 0.99)) if hit.any() else None,
            "hit_class_mismatch": int(np.sum(np.isfinite(a_aux[:, 0]) != np.isfinite(ref_aux[:, 0])))}
    return runs


PARETO_TOLERANCES = (1e-5, 1e-6, 1e-7, 1e-8, 1e-9)


def pareto_leg(local, reference_tol: float = 1e-10, c3_size: int = 2048) -> dict:
    """Accuracy against speed of FP32, mixed precision and FP64 (stated physics) on three scenes:
    the 1080p frame (c2) and draws 0 and 1 of the mixed-precision ablation at c3_size^2.  Each
    scene is first traced in FP64 at `reference_tol` (the converged image); then every precision
    at each tolerance of PARETO_TOLERANCES gives an event-timed trace (launch shape tuned once per
    scene and precision at tolerance 1e-6) and its per-pixel HDR error against the converged
    image (p99, p99.9, fraction above 1e-3; relative per pixel, floor 1e-6 x the image maximum).
    `at_equal_accuracy` lists, per scene and error target, the fastest tolerance of each
    precision whose p99 meets the target."""
    import torch

    import kerrtrace_b200 as kt
    from kerrtrace_b200 import autotune, workloads

    stream = torch.cuda.current_stream().cuda_stream
    scenes = [("c2", *workloads.scene("c2"))]
    for dr in (0, 1):
        c, cam = workloads.c3(dr, c3_size)
        scenes.append((f"c3_draw{dr}_{c3_size}", c, cam))
    precs = (("fp32", kt.PREC_FP32), ("mixed", kt.PREC_MIXED), ("fp64", kt.PREC_FP64))
    out = {"reference_tolerance": reference_tol, "tolerances": list(PARETO_TOLERANCES), "scenes": {}}
    for name, cfg0, cam in scenes:
        cfg0 = cfg0.copy()
        cfg0.mode = kt.MODE_SPEC
        n = cfg0.width * cfg0.height
        hdr = torch.zeros((n, 4), device="cuda")
        ref = torch.zeros((n, 4), device="cuda")
        err = torch.zeros(2, dtype=torch.int32, device="cuda")
        c = cfg0.copy()
        c.precision, c.tolerance = kt.PREC_FP64, reference_tol
        ctx = kt.Context(c, local)
        ctx.set_tuning(schedule=kt.SCHED_WAVEFRONT, blocks_per_sm=4)
        ctx.trace(cam, ref.data_ptr(), err.data_ptr(), stream, kt.SCHED_AUTO)
        torch.cuda.synchronize()
        ctx.close()
        r = ref[:, :3].double()
        floor = 1e-6 * float(r.abs().max())
        rows = []
        for pname, prec in precs:
            tuning = None
            for tol in PARETO_TOLERANCES:
                c = cfg0.copy()
                c.precision, c.tolerance = prec, tol
                ctx = kt.Context(c, local)
                if tuning is None:
                    t6 = cfg0.copy()
                    t6.precision, t6.tolerance = prec, 1e-6
                    tctx = kt.Context(t6, local)
                    tuning = autotune.autotune(tctx, cam, reps=1, stream=stream).best
                    tctx.close()
                ctx.set_tuning(**tuning)
                st = ctx.trace_counted(cam, hdr.data_ptr(), err.data_ptr(), stream, kt.SCHED_AUTO)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(2):
                    ctx.trace(cam, hdr.data_ptr(), err.data_ptr(), stream, kt.SCHED_AUTO)
                e1.record()
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / 2
                rel = ((hdr[:, :3].double() - r).abs() / r.abs().clamp_min(floor)).max(1).values
                q = torch.quantile(rel.float()[torch.randperm(n, device="cuda")[:min(n, 1 << 24)]],
                                   torch.tensor([0.99, 0.999], device="cuda"))
                rows.append({"precision": pname, "tolerance": tol, "trace_ms": round(ms, 4),
                             "mrays_s": round(n * c.spp / ms / 1e3, 1), "steps": int(st.steps),
                             "hdr_p99": float(q[0]), "hdr_p999": float(q[1]),
                             "hdr_frac_over_1e-3": float((rel > 1e-3).double().mean())})
                ctx.close()
        best = {}
        for target in (1e-4, 3e-5, 1e-5, 3e-6, 1e-6):
            best[f"p99<={target:g}"] = {}
            for pname, _ in precs:
                ok = [x for x in rows if x["precision"] == pname and x["hdr_p99"] <= target]
                f = min(ok, key=lambda x: x["trace_ms"]) if ok else None
                best[f"p99<={target:g}"][pname] = (
                    {"tolerance": f["tolerance"], "trace_ms": f["trace_ms"], "mrays_s": f["mrays_s"]} if f else None)
        out["scenes"][name] = {"size": f"{cfg0.width}x{cfg0.height}", "points": rows, "at_equal_accuracy": best}
    return out


def _log_hist(x, hist, lo: float = -12.0, bins: int = 1300):
    """Accumulate log10 of positive relative errors into 0.01-decade bins (zeros into bin 0)."""
    import torch
    v = torch.log10(x.clamp_min(10.0 ** lo))
    hist += torch.histc(v, bins=bins, min=lo, max=lo + bins / 100.0).double()


def _hist_quantile(hist, q: float, lo: float = -12.0):
    import torch
    c = torch.cumsum(hist, 0)
    if float(c[-1]) == 0:
        return None
    k = int(torch.searchsorted(c, q * c[-1]))
    return float(10.0 ** (lo + (k + 1) / 100.0))


def c3_leg(local, draws: int = 8, size: int = 4096) -> dict:
    """The ablation at the scene's tolerance (1e-6) and at the plain method's 1e-8."""
    return {"size": size, "runs": [c3_run(local, tol, draws, size) for tol in (1e-6, 1e-8)]}


def c3_run(local, tol: float, draws: int = 8, size: int = 4096) -> dict:
    """Mixed-precision ablation: 8 draws of (spin, inclination) seen at 4096^2 (FOV 20, r_obs
    60, stated physics, tolerance `tol`), each traced in FP64, FP32, mixed precision (compensated
    FP32 update, FP64 update inside 1.5 x the photon-orbit radius), mixed without the FP64 zone
    (`photon_zone_factor` 0.01, inside the horizon) and mixed with the FP64 update on the whole
    path (`photon_zone_factor` 1000).  Per variant: Mrays/s over all draws (event-timed trace kernel,
    launch shape tuned on draw 0); for the others the per-pixel relative error against the FP64
    run of HDR RGB and of the radius and redshift of the first disk crossing (max, p99, p99.9
    over all draws; quantiles from 0.01-decade histograms), the fraction of pixels above 1e-3
    and the hit/miss class mismatches."""
    import torch

    import kerrtrace_b200 as kt
    from kerrtrace_b200 import autotune, workloads

    n = size * size
    stream = torch.cuda.current_stream().cuda_stream
    precs = (("fp64", kt.PREC_FP64, 1.5), ("fp32", kt.PREC_FP32, 1.5), ("mixed", kt.PREC_MIXED, 1.5),
             ("mixed_no_zone", kt.PREC_MIXED, 0.01), ("mixed_whole_path", kt.PREC_MIXED, 1000.0))
    names = [p for p, _, _ in precs]
    hdr = {p: torch.zeros((n, 4), device="cuda") for p in names}
    aux = {p: torch.zeros((n, 4), device="cuda") for p in names}
    err = torch.zeros(2, dtype=torch.int32, device="cuda")
    tuning, ms_total, steps, zone = {}, {p: 0.0 for p in names}, {p: 0 for p in names}, {p: 0 for p in names}
    acc = {p: {"hist": {k: torch.zeros(1300, dtype=torch.float64, device="cuda") for k in ("hdr", "r", "g")},
               "max": {"hdr": 0.0, "r": 0.0, "g": 0.0}, "over": 0, "class": 0, "hits": 0} for p in names[1:]}
    per_draw = []
    for dr in range(draws):
        cfg, cam = workloads.c3(dr, size)
        cfg.tolerance = tol
        for pname, prec, zf in precs:
            c = cfg.copy()
            c.precision = prec
            c.photon_zone_factor = zf
            ctx = kt.Context(c, local)
            if dr == 0:
                tuning[pname] = autotune.autotune(ctx, cam, reps=1, stream=stream).best
            ctx.set_tuning(**tuning[pname])
            st = ctx.trace_counted(cam, hdr[pname].data_ptr(), err.data_ptr(), stream, kt.SCHED_AUTO,
                                   aux[pname].data_ptr())
            ctx.trace(cam, hdr[pname].data_ptr(), err.data_ptr(), stream, kt.SCHED_AUTO)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            ctx.trace(cam, hdr[pname].data_ptr(), err.data_ptr(), stream, kt.SCHED_AUTO)
            e1.record()
            torch.cuda.synchronize()
            ms_total[pname] += e0.elapsed_time(e1)
            steps[pname] += int(st.steps)
            zone[pname] += int(st.fp64_steps)
            ctx.close()
        ref = hdr["fp64"][:, :3].double()
        floor = 1e-6 * float(ref.abs().max())
        hit_ref = torch.isfinite(aux["fp64"][:, 0])
        row = {"spin": cfg.spin, "inclination_deg": workloads.c3_draws()[dr][1]}
        for pname in names[1:]:
            a = acc[pname]
            rel = ((hdr[pname][:, :3].double() - ref).abs() / ref.abs().clamp_min(floor)).max(1).values
            _log_hist(rel, a["hist"]["hdr"])
            a["max"]["hdr"] = max(a["max"]["hdr"], float(rel.max()))
            over = int((rel > 1e-3).sum())
            a["over"] += over
            hit = torch.isfinite(aux[pname][:, 0])
            cls = int((hit != hit_ref).sum())
            a["class"] += cls
            both = hit & hit_ref
            a["hits"] += int(both.sum())
            for k, col in (("r", 0), ("g", 1)):
                x = aux[pname][both, col].double()
                y = aux["fp64"][both, col].double()
                rk = (x - y).abs() / y.abs()
                _log_hist(rk, a["hist"][k])
                a["max"][k] = max(a["max"][k], float(rk.max()) if rk.numel() else 0.0)
            row[pname] = {"hdr_over_1e-3": over, "class_mismatch": cls}
        per_draw.append(row)
    out = {"tolerance": tol, "draws": per_draw, "tuning": tuning}
    for pname in names:
        out[pname] = {"mrays_s": round(draws * n / ms_total[pname] / 1e3, 1), "trace_ms_per_draw": round(ms_total[pname] / draws, 3),
                      "steps": steps[pname], "fp64_zone_steps": zone[pname]}
    for pname in names[1:]:
        a = acc[pname]
        e = {"pixels": draws * n, "hit_pixels_compared": a["hits"], "hdr_frac_over_1e-3": a["over"] / (draws * n),
             "hit_class_mismatch": a["class"]}
        for k, name in (("hdr", "hdr"), ("r", "r_cross"), ("g", "g")):
            e[f"{name}_max"] = a["max"][k]
            e[f"{name}_p99"] = _hist_quantile(a["hist"][k], 0.99)
            e[f"{name}_p999"] = _hist_quantile(a["hist"][k], 0.999)
        out[pname]["err_vs_fp64"] = e
    return out


def sequence_leg(cfg, tuning, local, moving: int = 60, resting: int = 30) -> dict:
    """Headless frame sequence through the app's loop (src/app.rs:141-198, 200-260): the c2
    observer orbits the hole by 0.5 degrees of azimuth per tick for `moving` ticks, then rests
    for `resting` ticks, when the re-render policy submits nothing.  Two frames in flight; each
    finished frame is handed back and the first one is written as PNG (app.rs:219-236).
    Reports frames rendered, ticks skipped, wall time, frames per second and Mrays/s."""
    import os
    import tempfile

    import kerrtrace_b200 as kt

    views = [kt.orbit_view(100.0, 85.0, 25.0, 0.5 * k) for k in range(moving)]
    views += [views[-1]] * resting
    r = kt.Renderer(cfg, local)
    r.set_tuning(tuning)
    state = kt.ViewState(views[0])
    png = os.path.join(tempfile.mkdtemp(prefix="kt_seq_"), "first_frame.png")
    rendered = skipped = done = 0
    first = None

    def hand_back(block: bool) -> bool:
        nonlocal done, first
        while True:
            f = r.ready_frame()
            if f is not None:
                if first is None:
                    first = f[1].copy()
                r.finish_frame(f[0])
                done += 1
                return True
            if not block:
                return False

    t0 = time.perf_counter()
    for v in views:
        if not state.should_render(v):
            skipped += 1
        while state.should_render(v):
            if r.submit_view(state, v):
                rendered += 1
                break
            hand_back(True)
        hand_back(False)
    while done < rendered:
        hand_back(True)
    wall = time.perf_counter() - t0
    r.close()
    written = kt.write_png(png, first, cfg.width, cfg.height)
    size = os.path.getsize(png)
    os.remove(png)
    os.rmdir(os.path.dirname(png))
    rays = rendered * cfg.width * cfg.height * cfg.spp
    return {"ticks": len(views), "frames_rendered": rendered, "ticks_skipped": skipped,
            "wall_ms": round(wall * 1e3, 2), "frames_per_s": round(rendered / wall, 1),
            "mrays_s": round(rays / wall / 1e6, 1), "first_frame_png_bytes": size if written else 0}


def batch_leg(local, reps: int, scale: int = 1) -> dict:
    """The batched-launch workload (64 renders: 16 each of 256^2, 512^2, 1024^2, 1920x1080 with
    random spins, inclinations, observer and disk radii): one batched launch in the shape the
    batch tuner picks (plain block shapes or the persistent launch), the same launch replayed from
    a CUDA graph, and the baseline of 64 sequential plain launches; then the same renders in
    stated physics and mixed precision."""
    import torch

    import kerrtrace_b200 as kt
    from kerrtrace_b200 import workloads

    jobs = workloads.c4_jobs(scale=scale)
    bufs = [(torch.zeros((c.width * c.height, 4), device="cuda"), torch.zeros(2, dtype=torch.int32, device="cuda"))
            for c, _ in jobs]
    b = kt.Batch([(c, cam, h.data_ptr(), e.data_ptr()) for (c, cam), (h, e) in zip(jobs, bufs)], local)
    rays = b.rays()
    stream = torch.cuda.current_stream().cuda_stream
    out = {"jobs": len(jobs), "rays": rays, "scale": scale}
    # launch shape of the batched launch: kt_batch_autotune (plain block shapes and the persistent
    # launch of job-uniform 32-pixel units), every candidate checked bit for bit
    rows = b.autotune(reps=2, stream=stream)
    out["tuner"] = [{"ms": round(ms, 3), **{k: t[k] for k in ("schedule", "block_x", "block_y", "blocks_per_sm")},
                     "identical": ok} for ms, t, ok in rows]
    out["tuning"] = b.tuning().as_dict()
    for name, fn in (("sequential_plain", lambda: b.trace_sequential(stream, kt.SCHED_PLAIN)),
                     ("batched_launch", lambda: b.trace(stream)),
                     ("batched_graph", lambda: b.trace_graph(stream))):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        out[name] = {"ms": round(ms, 3), "mrays_s": round(rays / ms / 1e3, 1)}
    out["speedup_graph_vs_sequential"] = round(out["sequential_plain"]["ms"] / out["batched_graph"]["ms"], 3)
    b.close()
    # the same 64 renders in stated physics and mixed precision, one graph-replayed launch
    mjobs = []
    for c, cam in jobs:
        c = c.copy()
        c.mode, c.precision = kt.MODE_SPEC, kt.PREC_MIXED
        mjobs.append((c, cam))
    mb = kt.Batch([(c, cam, h.data_ptr(), e.data_ptr()) for (c, cam), (h, e) in zip(mjobs, bufs)], local)
    out["mixed_tuner"] = [{"ms": round(ms, 3), **{k: t[k] for k in ("schedule", "block_x", "block_y", "blocks_per_sm")},
                           "identical": ok} for ms, t, ok in mb.autotune(reps=1, stream=stream)]
    mb.trace_graph(stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        mb.trace_graph(stream)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    out["mixed_batched_graph"] = {"ms": round(ms, 3), "mrays_s": round(mb.rays() / ms / 1e3, 1)}
    mb.close()
    return out


def adjoint_leg(local, reps: int, size: int = 512) -> dict:
    """The differentiable inverse problem (512^2, FOV 30, r_obs 50, stated physics): L2 loss on
    linear HDR between the image at the starting parameters and the target image; forward with
    step records, then the discrete adjoint (VJP) of the loss.  Per precision: forward, backward
    and adjoint Mrays/s (rays / (forward + backward)), the cost ratio, record memory and the
    gradient, and its agreement with central differences of the frozen-step model
    (Richardson-extrapolated, double images, unresolvable pixels masked; the FP32 records are
    replayed in FP64 arithmetic for them)."""
    import torch

    import kerrtrace_b200 as kt
    from kerrtrace_b200 import workloads

    n = size * size
    out = {"size": size, "rays": n, "theta_start": list(workloads.C5_START), "theta_target": list(workloads.C5_TARGET)}
    for pname, prec in (("fp32", kt.PREC_FP32), ("fp64", kt.PREC_FP64)):
        cfg, view = workloads.c5(size, prec)
        d = kt.Diff(cfg, view, device=local)
        err = torch.zeros(2, dtype=torch.int32, device="cuda")
        target = torch.zeros((n, 4), device="cuda")
        hdr = torch.zeros((n, 4), device="cuda")
        d.forward(list(workloads.C5_TARGET), target.data_ptr(), err.data_ptr())
        d.forward(list(workloads.C5_START), hdr.data_ptr(), err.data_ptr())
        torch.cuda.synchronize()
        w = 2.0 * (hdr - target)
        w[:, 3] = 0
        loss = float(((hdr[:, :3] - target[:, :3]).double() ** 2).sum())
        g = torch.zeros(4, dtype=torch.float64, device="cuda")
        tf, tb = [], []
        for _ in range(reps):
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record()
            d.forward(list(workloads.C5_START), hdr.data_ptr(), err.data_ptr())
            e1.record()
            d.backward(w.data_ptr(), g.data_ptr())
            e2.record()
            torch.cuda.synchronize()
            tf.append(e0.elapsed_time(e1))
            tb.append(e1.elapsed_time(e2))
        f_ms, b_ms = sorted(tf)[len(tf) // 2], sorted(tb)[len(tb) // 2]
        info = d.info()
        r = {"forward_ms": round(f_ms, 3), "backward_ms": round(b_ms, 3),
             "forward_mrays_s": round(n / f_ms / 1e3, 2), "adjoint_mrays_s": round(n / (f_ms + b_ms) / 1e3, 2),
             "cost_ratio": round((f_ms + b_ms) / f_ms, 2), "loss": loss, "grad": g.cpu().tolist(),
             "record_mb": round(info.record_bytes / 2**20, 2), "diff_device_mb": round(info.device_bytes / 2**20, 1),
             "overflow_rays": int(info.overflow_rays)}
        # central differences of the frozen-step model in double arithmetic: the FP64 records
        # replayed as they are, the FP32 records replayed in FP64 (kt_diff_replay_fp64)
        th = list(workloads.C5_START)
        eps = [1e-5, 1e-4, 1e-5, 1e-4]
        mask = torch.zeros(n, dtype=torch.bool, device="cuda")
        fd = []
        for j in range(4):
            img = {}
            for sgn in (1, -1):
                for k in (1, 2):
                    t2 = list(th)
                    t2[j] += sgn * eps[j] / k
                    hh = torch.zeros((n, 4), device="cuda")
                    h64 = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
                    fl = torch.zeros(n, dtype=torch.int32, device="cuda")
                    if prec == kt.PREC_FP64:
                        d.replay(t2, hh.data_ptr(), fl.data_ptr(), err.data_ptr(), hdr64_ptr=h64.data_ptr())
                    else:
                        d.replay_fp64(t2, h64.data_ptr(), fl.data_ptr(), err.data_ptr(), hh.data_ptr())
                    torch.cuda.synchronize()
                    img[(sgn, k)] = h64
                    mask |= fl.bool()
            f1 = (img[(1, 1)] - img[(-1, 1)]) / (2 * eps[j])
            f2 = (img[(1, 2)] - img[(-1, 2)]) / eps[j]
            mask |= ((f1 - f2).abs() > 1e-3 * f2.abs() + 1e-7 * f2.abs().max()).any(dim=1)
            fd.append((4 * f2 - f1) / 3)
        wm = w.clone()
        wm[mask] = 0
        d.backward(wm.data_ptr(), g.data_ptr())
        torch.cuda.synchronize()
        ga = g.cpu().tolist()
        ref = [float((fd[j] * wm[:, :3].double()).sum()) for j in range(4)]
        r["fd_check"] = {"eps": eps, "replay": "records as recorded" if prec == kt.PREC_FP64 else
                         "FP32 records replayed in FP64 arithmetic", "masked_pixels": int(mask.sum()),
                         "adjoint": ga, "central_differences": ref,
                         "rel_err": [abs(ga[j] - ref[j]) / max(abs(ref[j]), 1e-300) for j in range(4)]}
        if prec == kt.PREC_FP32:
            # the FP64 adjoint of the same FP32 records (kt_diff_backward_fp64): the model the
            # central differences above measure, differentiated in double
            d.backward_fp64(wm.data_ptr(), g.data_ptr())
            torch.cuda.synchronize()
            g64 = g.cpu().tolist()
            tb64 = []
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                d.backward_fp64(w.data_ptr(), g.data_ptr())
                e1.record()
                torch.cuda.synchronize()
                tb64.append(e0.elapsed_time(e1))
            b64 = sorted(tb64)[len(tb64) // 2]
            r["backward_fp64_records"] = {
                "backward_ms": round(b64, 3), "adjoint_mrays_s": round(n / (f_ms + b64) / 1e3, 2),
                "cost_ratio": round((f_ms + b64) / f_ms, 2), "adjoint": g64,
                "rel_err": [abs(g64[j] - ref[j]) / max(abs(ref[j]), 1e-300) for j in range(4)]}
        out[pname] = r
        d.close()
    return out


def run_ours(args, rank, world, local):
    import torch

    import kerrtrace_b200 as kt
    from kerrtrace_b200 import autotune, flops, workloads

    cfg, cam = rank_camera(workloads, args.workload, rank, world, args.size)
    cfg.mode = kt.MODE_SPEC if args.mode == "spec" else kt.MODE_REF
    cfg.precision = {"fp32": kt.PREC_FP32, "mixed": kt.PREC_MIXED, "fp64": kt.PREC_FP64}[args.precision]
    sched = {"auto": kt.SCHED_AUTO, "wavefront": kt.SCHED_WAVEFRONT, "plain": kt.SCHED_PLAIN}[args.schedule]
    ctx = kt.Context(cfg, local)
    n = cfg.width * cfg.height
    hdr = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    img = torch.zeros(n, dtype=torch.int32, device="cuda")
    err = torch.zeros(2, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    try:  # the FP32 roofline's denominator, measured on this GPU before the timed region
        measured_fma = kt.fma_peak(local, 16384)
    except kt.KtError:
        measured_fma = None
    if args.tuning:
        sc_, bx_, by_, bps_, rf_, od_ = (int(v) for v in args.tuning.split(","))
        ctx.set_tuning(schedule=sc_, block_x=bx_, block_y=by_, blocks_per_sm=bps_, refill_min=rf_, order=od_)
        sched = kt.SCHED_AUTO
        tuned = None
    else:
        tuned = autotune.autotune(ctx, cam, stream=stream) if sched == kt.SCHED_AUTO else None
    stats = ctx.trace_counted(cam, hdr.data_ptr(), err.data_ptr(), stream, sched)
    work = flops.trace_flops(stats)

    def step():
        err.zero_()
        ctx.trace(cam, hdr.data_ptr(), err.data_ptr(), stream, sched)
        ctx.post_fused(hdr.data_ptr(), img.data_ptr(), stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        for e0, e1, e2 in ev:
            flush.fill_(1.0)
            err.zero_()
            e0.record()
            ctx.trace(cam, hdr.data_ptr(), err.data_ptr(), stream, sched)
            e1.record()
            ctx.post_fused(hdr.data_ptr(), img.data_ptr(), stream)
            e2.record()
        torch.cuda.synchronize()
        barrier(world)
    clocks = clk.summary()
    t_steps = [a.elapsed_time(c) for a, _, c in ev]
    t_trace = [a.elapsed_time(b) for a, b, _ in ev]
    t_post = [b.elapsed_time(c) for _, b, c in ev]
    total_ms = max_over_ranks(sum(t_steps), world)
    rays_all = n * cfg.spp * world * args.steps
    value = job_mrays_s(n * cfg.spp * args.steps, world, total_ms)

    # end to end through the renderer API (host buffers), same launch shape
    rend = kt.Renderer(cfg, local)
    rend.set_schedule(sched)
    rend.set_tuning(ctx.tuning())
    cam_args = (list(cam.cam_pos), list(cam.fwd), list(cam.rgt), list(cam.up), cam.fov_scale)

    def frames(k):
        """k frames the way the reference host drives CudaRenderer: submit while a frame buffer
        is free (two in flight), poll ready_frame, hand each finished frame back."""
        submitted = done = 0
        while done < k:
            if submitted < k and rend.submit_render(*cam_args):
                submitted += 1
                continue
            got = rend.ready_frame()
            if got is not None:
                rend.finish_frame(got[0])
                done += 1

    frames(args.warmup)
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    frames(args.steps)
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    rend.close()
    e2e = {"value": round(rays_all / e2e_s / 1e6, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 52,
           "d2h_bytes_per_step": n * 4 + 8, "ms_per_step": round(e2e_s * 1e3 / args.steps, 4)}

    trace_ms = sum(t_trace) / len(t_trace)
    achieved = work / (trace_ms / 1e3) / 1e12
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    mhz = clocks.get("sm_mhz") or 1965.0
    nominal = sms * flops.FP32_LANES_PER_SM * 2 * mhz * 1e6 / 1e12
    peak = measured_fma[0] if measured_fma else nominal
    t = ctx.tuning()
    kernel = "trace_plain_kernel" if (t.schedule == kt.SCHED_PLAIN and sched == kt.SCHED_AUTO) or sched == kt.SCHED_PLAIN \
        else "trace_wavefront_kernel"
    roofline = {"bound": "fp32", "kernel": kernel,
                "achieved": round(achieved, 3), "peak": round(peak, 3), "unit": "TFLOP/s",
                "frac": round(achieved / peak, 4),
                "peak_source": ("measured: FP32 FMA throughput of this GPU (kt_fma_peak: 8 independent FMA "
                                f"chains per thread on every SM, best of 5 launches of {measured_fma[1]:.3f} ms)")
                if measured_fma else f"nominal: {sms} SMs x 128 lanes x 2 flops at the sampled clock",
                "nominal_at_clock": round(nominal, 3),
                "traffic": int(TRACE_TRAFFIC_PER_RAY * n * cfg.spp),
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one trace launch "
                                  "(c2 scene at 960x540: 149504 + 0 B), scaled to this launch by its rays",
                "trace_ms": round(trace_ms, 4),
                "post_ms": round(sum(t_post) / len(t_post), 4),
                "work": {"rays": int(stats.rays), "steps": int(stats.steps), "attempts": int(stats.attempts),
                         "rhs_evals": int(stats.rhs_evals), "frozen_rays": int(stats.frozen_rays),
                         "flops": work}}
    # trace (+ the pixel-ranking pass of a long-rays-first tuning) + bloom and post passes
    bloom_on = bool(cfg.bloom_enabled) and int(math.ceil(cfg.bloom_radius)) > 0 and cfg.bloom_intensity > 0
    launches_per_step = 1 + (1 if t.order == kt.ORDER_LONG_FIRST else 0) + (2 if bloom_on else 1)
    line = {
        "metric": "Mrays/s 1080p (c2 scene, trace + post)", "value": round(value, 3), "unit": "Mrays/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (procedural scene, camera rays)",
        "config": {"workload": workload_label(args.workload, cfg),
                   "schedule": args.schedule, "tuning": t.as_dict(),
                   "mode": "reference semantics (drop-in, bit-identical to the reference kernel)" if args.mode == "ref"
                   else "stated physics", "precision": args.precision,
                   "l2": "flushed between steps (256 MiB write outside the timed events)",
                   "parallelism": f"replica frames x{world}"},
        "e2e": e2e, "roofline": roofline, "clocks": clocks, "gpu_launches": launches_per_step * args.steps,
    }
    if tuned is not None:
        line["autotune"] = tuned.summary()
    # legs, each with the SM clock sampled while it runs; the long 4096^2 ablation goes last, so
    # that the heat it leaves does not lower the clocks of the shorter legs
    legs = [("retirement", args.no_retirement, lambda: retirement_leg(ctx, cfg, cam, stream)),
            ("precision", args.no_precision, lambda: precision_leg(cfg, cam, local, max(3, args.steps))),
            ("adjoint", args.no_adjoint, lambda: adjoint_leg(local, max(3, args.steps))),
            ("batch", args.no_batch, lambda: batch_leg(local, 3, args.batch_scale)),
            ("pareto", args.no_pareto, lambda: pareto_leg(local)),
            ("sequence", args.no_sequence, lambda: sequence_leg(cfg, ctx.tuning(), local)),
            ("c3", args.no_c3, lambda: c3_leg(local))]
    for name, skip, run in legs:
        if rank == 0 and world == 1 and not skip:
            with ClockSampler(local, period_s=0.02) as clk:
                line[name] = run()
            line[name]["clocks"] = clk.summary()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(cfg, cam, args.cpu_seconds)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()


def run_reference(args, rank, world, local):
    """The reference's own implementation of the path: its cuda/kernel.cu, compiled from source
    into oracle/_ref, launched like src/renderer/mod.rs:149-209.  Its scene values, KerrParams,
    LUTs and cameras come from the oracle's restatement of the reference host, so this process
    maps no product library."""
    import numpy as np
    import torch

    import oracle
    from kerrtrace_b200 import workloads

    if rank != 0:
        return
    host = oracle.Host()
    cfg, cam = rank_camera(workloads, args.workload, 0, 1, args.size, host=host)
    if not oracle.ref_lib_path(args.workload).exists():
        print(json.dumps({"impl": "reference", "unavailable": f"oracle/_ref/libktref_{args.workload}.so not built"}))
        return
    p, bb, disk = oracle.reference_inputs(cfg)
    ref = oracle.RefKernel(args.workload)
    ref.setup(p, bb, disk)
    n = cfg.width * cfg.height
    hdr = torch.zeros((n, 4), device="cuda")
    bloom = torch.zeros((n, 4), device="cuda")
    img = torch.zeros(n, dtype=torch.int32, device="cuda")
    err = torch.zeros(2, dtype=torch.int32, device="cuda")
    host_img = torch.zeros(n, dtype=torch.int32).pin_memory()
    host_err = torch.zeros(2, dtype=torch.int32).pin_memory()
    radius = int(math.ceil(np.float32(cfg.bloom_radius))) if cfg.bloom_radius > 0 else 0
    sigma = float(np.float32(cfg.bloom_radius) / np.float32(3.0))
    active = int(bool(cfg.bloom_enabled) and radius > 0 and cfg.bloom_intensity > 0)

    def frame():  # src/renderer/mod.rs:149-209
        err.zero_()
        ref.trace(hdr.data_ptr(), cfg, cam, cfg.lut_max_temp, err.data_ptr(), p.disk_inner)
        host_err.copy_(err, non_blocking=True)
        if active:
            ref.bloom(hdr.data_ptr(), bloom.data_ptr(), cfg, radius, sigma, active)
        ref.post(hdr.data_ptr(), bloom.data_ptr(), img.data_ptr(), cfg, radius, sigma, cfg.bloom_intensity, active)
        host_img.copy_(img, non_blocking=True)

    for _ in range(args.warmup):
        frame()
    torch.cuda.synchronize()
    evs = []
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            frame()
            e1.record()
            evs.append((e0, e1))
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    dev_ms = sum(a.elapsed_time(b) for a, b in evs)
    rays = n * cfg.spp * args.steps
    value = rays / (dev_ms / 1e3) / 1e6
    line = {"impl": "reference", "metric": "Mrays/s 1080p (c2 scene, trace + post)", "value": round(value, 3),
            "unit": "Mrays/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(dev_ms / args.steps, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (procedural scene, camera rays)",
            "config": {"workload": workload_label(args.workload, cfg),
                       "implementation": "reference cuda/kernel.cu compiled from source for sm_100a "
                                         "(-use_fast_math, the reference's #define header), mod.rs launch sequence"},
            "e2e": {"value": round(rays / wall / 1e6, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 52,
                    "d2h_bytes_per_step": n * 4 + 8},
            "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s", "cores": 0, "kind": "reference",
                             "sample": "the reference's path has no CPU implementation: this line times its GPU "
                                       "kernels (oracle/_ref) on the same B200"},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    ref.close()


def main():
    args = parse()
    rank, world, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, rank, world, local)
        else:
            run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
