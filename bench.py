"""Benchmark: Mrays/s of the plain wavefront path tracer on the 1M-triangle scene,
plus the same frame with SVO path guiding (WFPGTracer) and the equal-time MSE
of both against a converged plain render (the "guided" object of the line).

Workload ("clusters-1M"): 1000 Gaussian clusters x 1000 triangles (seed 1),
1920x1080, 1 sample per pixel per step ("Samples": 1), depth 8, NEE on,
Russian roulette from depth 3, samples splatted through a Tent filter of
radius 1 pixel (the reference's tracer configurations).  One step = one
frame: camera rays + 8 trace/partition/shade depths + the filter splat,
replayed from a captured CUDA graph.
Rays traced = camera + path + NEE rays entering the traversal, summed over
depths (the reference's "rays entering HitRays").

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torch.distributed (one process per GPU) as independent
replicas: each rank renders its own frames of the same workload (weak
scaling; the path tracer has no exchange step).  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import dataclasses
import datetime
import math
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mrays/s"
WORKLOAD = {"workload": "clusters-1M plain path tracing", "triangles": 1000008,
            "resolution": "1920x1080", "spp_per_step": 1, "max_depth": 8,
            "nee": True, "rr_start": 3, "scene_seed": 1,
            "recon_filter": "Tent, radius 1 pixel (the reference's tConf filter)",
            "l2": "inputs larger than L2 (ray/hit buffers ~470 MB, BVH ~180 MB)"}
# committed ncu summaries of the traversal kernel, per traversal mode
TRACE_PROFILE = {0: "k_trace_clusters1M_bvh2.md", 1: "k_trace_wide_clusters1M.md"}
OPTS = {"Samples": 1, "MaxDepth": 8, "NextEventEstimation": 1, "RussianRouletteStart": 3,
        "DirectLightMIS": 0}
# FilterOptions of the reference's tracer configurations (tConf_veach_*.json)
RECON = {"type": "Tent", "radius": 1.0}


def _attach_filter(system, t):
    t.attach_recon_filter(system.generate_recon_filter(RECON))


def _traffic_per_launch(traversal):
    """DRAM bytes per traversal launch from the committed ncu summary."""
    import re
    f = ROOT / "profiles" / TRACE_PROFILE[traversal]
    if not f.exists():
        return None
    m = re.search(r"dram_bytes_per_launch \(mean of \d+\): (\d+)", f.read_text())
    return int(m.group(1)) if m else None


# Algorithmic bytes of the traversal (per unit): per ray 72 B (ray 32 + id 4
# + key 4 in; tMax 4 + key 4 + transform 4 + primitive 8 + barycentrics 8 +
# status 4 out), per node visited its node bytes (8-wide quantised 80 B,
# binary LBVH 64 B), per triangle tested 36 B (three vertices).
RAY_BYTES, TRI_BYTES = 72, 36
NODE_BYTES = {0: 64, 1: 80}


def trace_bytes(rays: float, visits: float, tris: float, traversal: int) -> float:
    return RAY_BYTES * rays + NODE_BYTES[traversal] * visits + TRI_BYTES * tris


def _trace_roofline(t, prof: dict, traversal: int, traffic, peak: float,
                    peak_kind: str) -> dict:
    """Roofline of the traversal kernels over one profiled frame: the
    algorithmic bytes of the frame's rays, node visits and triangle tests
    (counted by the counting form of the kernels the frame runs) over the
    frame's traversal time."""
    tb = trace_bytes(prof["rays"], prof["node_visits"], prof["tri_tests"], traversal)
    ts = prof["trace_ms"] / 1e3
    achieved = tb / ts / 1e9 if ts > 0 else 0.0
    return {"bound": "hbm",
            "kernel": "k_trace_wide / k_trace_wide_refill" if traversal == 1 else "k_trace",
            "kernel_per_depth": t.wide_orders() if traversal == 1 else None,
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "peak_kind": peak_kind,
            "algorithmic_bytes_per_frame": tb, "rays_per_frame": prof["rays"],
            "trace_ms_per_frame": prof["trace_ms"],
            "launches_per_frame": prof.get("trace_launches"),
            "node_visits_per_ray": prof["node_visits"] / max(prof["rays"], 1),
            "tri_tests_per_ray": prof["tri_tests"] / max(prof["rays"], 1)}


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self._t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def aggregate_ranks(dist, torch, ms: float, e2e_ms: float, rays: int, e2e_rays: int,
                    device: str):
    """Whole-job figures of the replicas: the slowest rank's times (the job
    ends when its last replica does) and the sum of every rank's rays."""
    tt = torch.tensor([ms, e2e_ms], dtype=torch.float64, device=device)
    rr = torch.tensor([rays, e2e_rays], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    dist.all_reduce(rr, op=dist.ReduceOp.SUM)
    return float(tt[0]), float(tt[1]), int(rr[0]), int(rr[1])


def run_ours(args, rank: int, world: int, dist) -> dict | None:
    import torch
    import meturay_b200 as m

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    scene = m.scenes.clusters(seed=1, width=args.res[0], height=args.res[1])
    system = m.TracerSystem(dev)
    g = m.GPUScene(system, scene)
    g.set_wide_order(args.wide_order)
    g.set_wide_collapse(args.wide_collapse)
    g.construct_accelerators()
    g.set_traversal(args.traversal)
    if args.only == "guided":
        return run_guided(args, g, m, torch, dev)
    if args.only == "learned":
        return {"learned": run_learned(args, m, system, torch)}
    if args.only == "closed":
        return {"closed_scene": run_closed(args, m, system, torch)}
    t = m.PathTracer(system, g)
    t.set_options(dict(OPTS, Seed=1 + rank))
    _attach_filter(system, t)
    stream = torch.cuda.ExternalStream(t.stream)

    for _ in range(args.warmup):
        t.render_frame()
    torch.cuda.synchronize()
    rays0, _ = t.stats()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        t.render_frame()
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    rays1, _ = t.stats()
    rays = rays1 - rays0

    # ---- end to end through the public API with host buffers ----
    import ctypes as C
    img_bytes = scene.width * scene.height * 16
    host_img = torch.empty(scene.width * scene.height * 4, dtype=torch.float32).pin_memory()
    cam_bytes = 56  # the pinhole frame uploaded by set_camera
    for _ in range(2):
        t.set_camera(scene.camera)
        t.render_frame()
        t.image_into(C.c_void_p(host_img.data_ptr()))
    torch.cuda.synchronize()
    r0, _ = t.stats()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(args.steps):
        t.set_camera(scene.camera)
        t.render_frame()
        # pipelined read-back: this frame's image is snapshotted on the device
        # and copied to pinned host memory while the next frame renders
        t.image_into_async(C.c_void_p(host_img.data_ptr()))
    t.wait_image()          # the last copy is inside the timed region
    s1.record(stream)
    s1.synchronize()
    e2e_ms = s0.elapsed_time(s1)
    r1, _ = t.stats()
    e2e_rays = r1 - r0

    # ---- roofline of the traversal kernel (one stepwise profiled frame) ----
    prof = t.profile_frame()
    launches = t.launches_per_frame() * args.steps
    guided = run_guided(args, g, m, torch, dev) \
        if (args.guided and args.only == "all" and rank == 0 and world == 1) else None
    batching = serving = None
    if args.pool and args.only == "all" and rank == 0 and world == 1:
        batching = run_batching(args, m, system, torch)
        if not args.pool_block:
            args.pool_block = batching["autotune"]["chosen"]["block"]
            args.pool_stack = batching["autotune"]["chosen"]["stack"]
        serving = run_serving(args, m, system)
    learned = run_learned(args, m, system, torch) \
        if (args.learned and args.only == "all" and rank == 0 and world == 1) else None
    closed = run_closed(args, m, system, torch) \
        if (args.closed and args.only == "all" and rank == 0 and world == 1) else None

    if dist:
        ms, e2e_ms, rays, e2e_rays = aggregate_ranks(dist, torch, ms, e2e_ms, rays, e2e_rays,
                                                     "cuda")
    if rank != 0:
        return None

    peak, peak_kind = _peaks()
    roof = _trace_roofline(t, prof, args.traversal, _traffic_per_launch(args.traversal), peak,
                           peak_kind)
    roof["wide_collapse"] = g.wide_collapse()
    roof["stage_ms"] = {k: prof[k] for k in ("camera_ms", "trace_ms", "partition_ms", "shade_ms",
                                             "resolve_ms")}
    return {
        "metric": METRIC,
        "value": rays / (ms / 1e3) / 1e6,
        "unit": "Mrays/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded clusters-1M scene)",
        "config": run_config(world),
        "traversal": "8-wide quantised BVH" if args.traversal else "binary LBVH",
        "rays_per_step": rays / args.steps / world,
        "mpaths_per_s": scene.width * scene.height * world * args.steps / ms / 1e3,
        "e2e": {"value": e2e_rays / (e2e_ms / 1e3) / 1e6, "unit": "Mrays/s",
                "h2d_bytes_per_step": cam_bytes, "d2h_bytes_per_step": img_bytes},
        "roofline": roof,
        "gpu_launches": launches,
        "clocks": clk,
        "guided": guided,
        "closed_scene": closed,
        "batching": batching,
        "serving": serving,
        "learned": learned,
    }


# WFPG options of the guided run (WFPGTracer.h:25-96; tConf_veach_product.json
# values for the ones the config does not fix): leaf depth 10, field
# 64^2 for the first two depths then 32^2, 16^2, 8^2 (WFPGTracer.cu:224-230)
GUIDED_OPTS = dict(OPTS, OctreeLevel=10, MinRayBinLevel=5, BinRayCount=512,
                   DoProductPathGuiding=1, GuideBounceAmount=512)
GUIDED_FLOATS = {"BXDF-GuideMISRatio": 0.5, "RFieldFilterAlpha": 0.6}


def _frames_image(t, frames: int) -> np.ndarray:
    """rgb / w after `frames` frames (w: the filter's weight sum per pixel)."""
    t.reset_image()
    for _ in range(frames):
        t.render_frame()
    img = t.image().astype(np.float64)
    w = img[..., 3:]
    return np.where(w > 0, img[..., :3] / np.where(w > 0, w, 1.0), 0.0)


def _budget_image(t, budget_ms: float, est_ms: float, torch):
    """rgb / w after as many frames as fit in `budget_ms` of device time on
    the tracer's stream, cold start (octree build, warm-up frames) included;
    frames run in chunks bracketed by CUDA events.  Returns (image, frames,
    device ms used)."""
    t.reset_image()
    stream = torch.cuda.ExternalStream(t.stream)
    used, frames, est = 0.0, 0, max(est_ms, 1e-3)
    while budget_ms - used > 0.5 * est:
        k = max(1, int(0.5 * (budget_ms - used) / est))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            t.render_frame()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        used += ms
        frames += k
        est = max(ms / k, 1e-3)
    img = t.image().astype(np.float64)
    w = img[..., 3:]
    return np.where(w > 0, img[..., :3] / np.where(w > 0, w, 1.0), 0.0), frames, used


def _reference(make, frames: int):
    """A converged render as two independent halves: (their average, the
    variance of that average per pixel and channel, estimated as
    mean((R1 - R2)^2) / 4, and the same for the relative error).  The
    variance is the floor every error against the reference carries;
    subtracting it leaves the run's own error."""
    halves = []
    for seed in (0, 1):
        t = make(seed)
        halves.append(_frames_image(t, max(1, frames // 2)))
        t.close()
    r1, r2 = halves
    ref = 0.5 * (r1 + r2)
    d2 = (r1 - r2) ** 2
    return ref, float(np.mean(d2)) / 4.0, float(np.mean(d2 / (ref * ref + 0.01))) / 4.0


def _clamped_mse(img, ref) -> float:
    """MSE after clamping both images at the reference's 99.9th percentile:
    a score that a single firefly pixel cannot dominate (it is biased, so
    it only ranks samplers; it is not an error estimate)."""
    c = float(np.percentile(ref, 99.9))
    return float(np.mean((np.minimum(img, c) - np.minimum(ref, c)) ** 2))


def _rel_mse(img, ref) -> float:
    """Relative MSE, mean((x - r)^2 / (r^2 + 0.01)): bright outliers weigh
    less than in the MSE, so it moves less with rare high-energy paths."""
    return float(np.mean((img - ref) ** 2 / (ref * ref + 0.01)))


def run_guided(args, g, m, torch, dev: int) -> dict:
    """The same frame with SVO path guiding, and the equal-time MSE of the
    guided and plain tracers against a converged plain render
    (Python/mse_hdr.py:36-44: mean over pixels and RGB of the squared
    difference)."""
    t = m.WFPGTracer(g.system, g)
    t.set_options(dict(GUIDED_OPTS, Seed=101))
    t.set_options(GUIDED_FLOATS)
    _attach_filter(g.system, t)
    stream = torch.cuda.ExternalStream(t.stream)
    for _ in range(args.warmup):
        t.render_frame()
    torch.cuda.synchronize()
    steps = max(10, args.steps // 5)
    r0, _ = t.stats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        t.render_frame()
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    r1, _ = t.stats()
    guided_ms = ms / steps
    stages = [t.profile_stages() for _ in range(3)]
    out = {"metric": METRIC, "value": (r1 - r0) / (ms / 1e3) / 1e6, "unit": "Mrays/s",
           "steps": steps, "ms_per_step": guided_ms,
           "rays_per_step": (r1 - r0) / steps,
           "launches_per_frame": t.launches_per_frame(),
           "stage_ms": {k: float(np.mean([x[k] for x in stages]))
                        for k in stages[0] if k.endswith("_ms")},
           "config": {"tracer": "WFPGTracer", **{k: v for k, v in GUIDED_OPTS.items()},
                      **GUIDED_FLOATS,
                      "field": "64x64 at depths 0-1, then 32x32, 16x16, 8x8",
                      "leaf_radiance": "64-bit fixed-point sums (2^-24), FP16 averages"}}
    if args.mse_budget_ms <= 0:
        return out
    # ---- equal-time MSE ----
    # The converged render is the plain tracer with NEE and MIS (the same
    # expectation as every estimator below, at far lower variance: NEE
    # without MIS throws fireflies off glossy lobes and next to the lights,
    # which would make a reference of that estimator noisier than the runs
    # it scores).
    def make_ref(half):
        r = m.PathTracer(g.system, g)
        r.set_options(dict(OPTS, DirectLightMIS=1, Seed=99 + 1000 * half))
        _attach_filter(g.system, r)
        return r
    ref_img, ref_var, ref_rvar = _reference(make_ref, args.mse_reference_spp)
    budget = float(args.mse_budget_ms)

    def run(kind, opts, floats, seed):
        def make(sd):
            t = (m.PathTracer if kind == "plain" else m.WFPGTracer)(g.system, g)
            t.set_options(dict(opts, Seed=sd))
            if floats:
                t.set_options(floats)
            _attach_filter(g.system, t)
            return t
        probe = make(seed + 500)
        for _ in range(5):
            probe.render_frame()
        est = _frame_ms(probe, torch, frames=10)
        probe.close()
        t = make(seed)   # a cold start: the octree build counts against the budget
        img, frames, used = _budget_image(t, budget, est, torch)
        t.close()
        raw = float(np.mean((img - ref_img) ** 2))
        return {"frames": frames, "ms_per_frame": est, "device_ms": used,
                "mse": raw - ref_var, "mse_raw": raw, "mse_x_frames": (raw - ref_var) * frames,
                "rel_mse": _rel_mse(img, ref_img) - ref_rvar,
                "clamped_mse": _clamped_mse(img, ref_img)}

    mis = {"DirectLightMIS": 1}
    nonee = {"NextEventEstimation": 0}
    runs = {
        # the configured options (the reference's defaults: NEE, no MIS)
        "plain": ("plain", OPTS, None),
        "guided": ("wfpg", GUIDED_OPTS, GUIDED_FLOATS),
        "wfpg_unguided": ("wfpg", dict(GUIDED_OPTS, SkipPG=1), GUIDED_FLOATS),
        # NEE with MIS (the plain tracer only: with MIS the guided tracers
        # are biased, the NEE weight using the BxDF pdf and the guided path
        # ray the mixture pdf, WFPGTracerKC.cuh:338-347)
        "plain_mis": ("plain", dict(OPTS, **mis), None),
        # NEE off, as the reference's own WFPG configurations run
        # (WorkingDir/tConf_veach_product.json)
        "plain_nonee": ("plain", dict(OPTS, **nonee), None),
        "guided_nonee": ("wfpg", dict(GUIDED_OPTS, **nonee), GUIDED_FLOATS),
        "guided_nonee_bounce1": ("wfpg", dict(GUIDED_OPTS, GuideBounceAmount=1, **nonee),
                                 GUIDED_FLOATS),
    }
    res = {k: run(kind, o, f, 7 + i) for i, (k, (kind, o, f)) in enumerate(runs.items())}

    def ratio(a, b):
        return res[a]["mse"] / res[b]["mse"] if res[b]["mse"] > 0 else None

    out["equal_time_mse"] = {
        "budget_ms": budget, "reference_spp": args.mse_reference_spp,
        "reference": "plain tracer, NEE with MIS, two halves of other seeds",
        "reference_variance": ref_var, **res,
        "guided_over_plain": ratio("guided", "plain"),
        "guided_over_wfpg_unguided": ratio("guided", "wfpg_unguided"),
        "guided_nonee_over_plain_nonee": ratio("guided_nonee", "plain_nonee"),
        "note": "1 spp per frame at 1920x1080; every MSE less the reference's own variance "
                "(mse_raw keeps it); mse_x_frames is the error per frame of samples; guided "
                "tracers start with a cold octree, whose build counts against the budget "
                "(device time)"}
    return out
    # ---- equal-time MSE ----
    p = m.PathTracer(g.system, g)
    p.set_options(dict(OPTS, Seed=7))
    _attach_filter(g.system, p)
    for _ in range(2):
        p.render_frame()
    torch.cuda.synchronize()
    pstream = torch.cuda.ExternalStream(p.stream)
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record(pstream)
    for _ in range(20):
        p.render_frame()
    q1.record(pstream)
    q1.synchronize()
    plain_ms = q0.elapsed_time(q1) / 20
    def make_ref(half):
        r = m.PathTracer(g.system, g)
        r.set_options(dict(OPTS, Seed=99 + 1000 * half))
        _attach_filter(g.system, r)
        return r
    ref_img, ref_var, ref_rvar = _reference(make_ref, args.mse_reference_spp)
    budget = float(args.mse_budget_ms)
    plain_img, plain_frames, plain_used = _budget_image(p, budget, plain_ms, torch)
    gt = m.WFPGTracer(g.system, g)   # a cold cache: learning is part of the budget
    gt.set_options(dict(GUIDED_OPTS, Seed=202))
    gt.set_options(GUIDED_FLOATS)
    _attach_filter(g.system, gt)
    guided_img, guided_frames, guided_used = _budget_image(gt, budget, guided_ms, torch)
    # the same guider with coarser ray bins (MinRayBinLevel 3, BinRayCount
    # 4096): fewer radiance fields per wavefront, each shared by more rays
    coarse = dict(GUIDED_OPTS, MinRayBinLevel=3, BinRayCount=4096)
    gc = m.WFPGTracer(g.system, g)
    gc.set_options(dict(coarse, Seed=101))
    gc.set_options(GUIDED_FLOATS)
    _attach_filter(g.system, gc)
    for _ in range(3):
        gc.render_frame()
    gc_ms = _frame_ms(gc, torch, frames=10)
    gc.close()
    gc = m.WFPGTracer(g.system, g)
    gc.set_options(dict(coarse, Seed=202))
    gc.set_options(GUIDED_FLOATS)
    _attach_filter(g.system, gc)
    coarse_img, coarse_frames, coarse_used = _budget_image(gc, budget, gc_ms, torch)
    gc.close()
    raw_c = float(np.mean((coarse_img - ref_img) ** 2))
    raw_p = float(np.mean((plain_img - ref_img) ** 2))
    raw_g = float(np.mean((guided_img - ref_img) ** 2))
    mse_p, mse_g = raw_p - ref_var, raw_g - ref_var
    out["equal_time_mse"] = {
        "budget_ms": budget, "reference_spp": args.mse_reference_spp,
        "reference_variance": ref_var,
        "plain": {"frames": plain_frames, "ms_per_frame": plain_ms, "device_ms": plain_used,
                  "mse": mse_p, "mse_raw": raw_p,
                  "rel_mse": _rel_mse(plain_img, ref_img) - ref_rvar,
                  "clamped_mse": _clamped_mse(plain_img, ref_img)},
        "guided": {"frames": guided_frames, "ms_per_frame": guided_ms,
                   "device_ms": guided_used, "mse": mse_g, "mse_raw": raw_g,
                   "rel_mse": _rel_mse(guided_img, ref_img) - ref_rvar,
                   "clamped_mse": _clamped_mse(guided_img, ref_img)},
        "guided_coarse_bins": {"MinRayBinLevel": 3, "BinRayCount": 4096,
                               "frames": coarse_frames, "ms_per_frame": gc_ms,
                               "device_ms": coarse_used, "mse": raw_c - ref_var,
                               "mse_raw": raw_c,
                               "rel_mse": _rel_mse(coarse_img, ref_img) - ref_rvar,
                               "clamped_mse": _clamped_mse(coarse_img, ref_img)},
        "guided_over_plain": mse_g / mse_p if mse_p > 0 else None,
        "mse_x_frames": {"plain": mse_p * plain_frames, "guided": mse_g * guided_frames},
        "note": "1 spp per frame at 1920x1080; the reference is two separate plain renders "
                "(other seeds), whose own variance is subtracted from every MSE (mse_raw keeps "
                "it); the guided tracer starts with a cold octree, and its build and every "
                "frame count against the budget (device time)"}
    return out


# ---- bounce-heavy closed scene -------------------------------------------
CLOSED = {"Samples": 4, "MaxDepth": 5, "NextEventEstimation": 1, "RussianRouletteStart": 3,
          "DirectLightMIS": 0}
STAGES5 = ("camera_ms", "trace_ms", "partition_ms", "shade_ms", "resolve_ms")


def run_closed(args, m, system, torch) -> dict:
    """The plain tracer on a closed scene at a resolution that fills the GPU:
    the Cornell box (seed 1, 7,692 triangles) at 1920x1080, 4 spp per frame,
    depth 5, NEE, Tent filter.  Every camera ray hits and most paths bounce
    to the last depth, so partition, shading and incoherent secondary rays
    carry the frame; reported with its stage split and traversal roofline."""
    scene = m.scenes.cornell(seed=1, width=1920, height=1080)
    g = m.GPUScene(system, scene)
    g.set_wide_collapse(args.wide_collapse)
    g.construct_accelerators()
    g.set_traversal(args.traversal)
    t = m.PathTracer(system, g)
    t.set_options(dict(CLOSED, Seed=5))
    _attach_filter(system, t)
    stream = torch.cuda.ExternalStream(t.stream)
    for _ in range(max(3, args.warmup)):
        t.render_frame()
    torch.cuda.synchronize()
    steps = max(5, min(args.steps, 20))
    r0, _ = t.stats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        t.render_frame()
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    r1, _ = t.stats()
    profs = [t.profile_frame() for _ in range(3)]
    prof = {k: float(np.mean([x[k] for x in profs])) for k in profs[0]}
    peak, peak_kind = _peaks()
    roof = _trace_roofline(t, prof, args.traversal, None, peak, peak_kind)
    roof["wide_collapse"] = g.wide_collapse()
    total = sum(prof[k] for k in STAGES5)
    out = {"metric": METRIC, "value": (r1 - r0) / (ms / 1e3) / 1e6, "unit": "Mrays/s",
           "steps": steps, "ms_per_step": ms / steps, "rays_per_step": (r1 - r0) / steps,
           "camera_rays_per_step": scene.width * scene.height * CLOSED["Samples"],
           "stage_ms": {k: prof[k] for k in STAGES5},
           "stage_share": {k: prof[k] / total for k in STAGES5},
           "roofline": roof,
           "config": {"scene": "Cornell box (seed 1), 7,692 triangles", "resolution": "1920x1080",
                      **CLOSED, "recon_filter": "Tent, radius 1 pixel"}}
    t.close()
    return out


# ---- wavefront pool: batching (many small scenes) and serving ----------
BATCH = {"scenes": 256, "tris": (1000, 64000), "res": (64, 128, 256, 512), "spp": 16,
         "max_depth": 6, "seed": 3}
SERVE = {"scenes": 32, "tris": (10000, 2000000), "res": (256, 512, 1024),
         "spp": (1, 16, 64), "rate_per_s": 200.0, "max_depth": 5, "seed": 4}


def _log_uniform(rng, lo, hi):
    return int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))


def _pool_scenes(m, system, rng, n, tris):
    """n seeded Cornell-style scenes (the 8k-triangle Cornell generator), triangle counts
    log-uniform in `tris` through the spheres' tessellation."""
    out = []
    for i in range(n):
        t = _log_uniform(rng, *tris)
        sc = m.scenes.cornell(seed=10_000 + i, triangles=t, width=64, height=64)
        g = m.GPUScene(system, sc)
        g.construct_accelerators()
        out.append(g)
    return out


def run_batching(args, m, system, torch) -> dict:
    """Batching: one frame of 16 spp for each of 256 seeded scenes, all jobs in one
    wavefront pool (every traversal launch covers every scene in flight);
    wavefront size and traversal launch shape picked by the autotuner."""
    from meturay_b200.pool import autotune
    rng = np.random.default_rng(BATCH["seed"])
    scenes = _pool_scenes(m, system, rng, BATCH["scenes"], BATCH["tris"])
    jobs = []
    for i, g in enumerate(scenes):
        r = int(rng.choice(BATCH["res"]))
        jobs.append(m.Job(g, r, r, samples=1, frames=BATCH["spp"], max_depth=BATCH["max_depth"],
                          seed=100 + i))
    largest = max(j.width * j.height for j in jobs)
    # the autotuner's sample: one frame of every fourth job; wavefront sizes
    # of 2^16 .. 2^22 rays (two rays per camera sample)
    caps = [1 << k for k in (15, 17, 19, 21)]
    tune = autotune(system, [dataclasses.replace(j, frames=1) for j in jobs[::4]],
                    capacities=caps, blocks=(64, 128, 256), stacks=(64, 128, 0),
                    max_depth=BATCH["max_depth"], iterations=3)
    feasible = [r for r in tune["table"] if r["capacity"] >= largest]
    best = max(feasible, key=lambda r: r["mrays_s"])
    pool = m.WavefrontPool(system, capacity=best["capacity"], max_depth=BATCH["max_depth"])
    pool.set_launch(best["block"], best["stack"])
    pool.run([dataclasses.replace(j, frames=1) for j in jobs[:8]])  # graph capture, warm-up
    stream = torch.cuda.ExternalStream(lib_stream(pool))
    r0 = pool.stats()["rays"]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    t0 = time.perf_counter()
    pool.run(jobs)
    e1.record(stream)
    e1.synchronize()
    wall = time.perf_counter() - t0
    ms = e0.elapsed_time(e1)
    st = pool.stats()
    rays = st["rays"] - r0
    samples = sum(j.width * j.height * j.frames for j in jobs)
    pool.close()
    return {"metric": METRIC, "value": rays / (ms / 1e3) / 1e6, "unit": "Mrays/s",
            "seconds": ms / 1e3, "wall_seconds": wall, "rays": rays, "samples": samples,
            "jobs": len(jobs), "triangles_total": int(sum(g.scene.triangle_count for g in scenes)),
            "config": {**BATCH, "wavefront": "one pool; every traversal launch covers all "
                                             "scenes in flight; iterations replay one graph"},
            "autotune": {"chosen": best, "table": tune["table"],
                         "note": "capacity = camera samples per iteration (2 rays each); "
                                 "measured on every fourth job, 3 iterations each"}}


def lib_stream(pool):
    from meturay_b200._lib import lib
    return lib.mrb_pool_stream(pool._h)


def _sphere_camera(rng, center, radius):
    u = rng.normal(size=3)
    u /= np.linalg.norm(u)
    pos = np.asarray(center) + radius * u
    up = [0.0, 1.0, 0.0] if abs(u[1]) < 0.95 else [1.0, 0.0, 0.0]
    fov = math.radians(40.0)
    return {"position": pos.tolist(), "gaze": list(center), "up": up,
            "near_far": [0.01, 100.0], "fov": [fov, fov]}


def run_serving(args, m, system) -> dict:
    """Serving: Poisson arrivals of render jobs against one wavefront pool with
    32 resident scenes; jobs are admitted by free HBM and join the running
    iterations as they arrive.  Latency = arrival to the end of the
    iteration that finished the job (host clock)."""
    from meturay_b200.pool import serve
    rng = np.random.default_rng(SERVE["seed"])
    scenes = _pool_scenes(m, system, rng, SERVE["scenes"], SERVE["tris"])
    n = int(args.serve_jobs)
    t, arrivals = 0.0, []
    for i in range(n):
        t += float(rng.exponential(1.0 / SERVE["rate_per_s"]))
        g = scenes[int(rng.integers(len(scenes)))]
        r = int(rng.choice(SERVE["res"]))
        spp = int(rng.choice(SERVE["spp"]))
        job = m.Job(g, r, r, samples=1, frames=spp, max_depth=SERVE["max_depth"],
                    seed=1000 + i, camera=_sphere_camera(rng, (0.5, 0.5, 0.5), 2.0),
                    meta={"spp": spp})
        arrivals.append((t, job))
    pool = m.WavefrontPool(system, capacity=1 << 21, max_depth=SERVE["max_depth"])
    if args.pool_block:
        pool.set_launch(args.pool_block, args.pool_stack)
    pool.run([dataclasses.replace(arrivals[0][1], frames=1)])  # graph capture, warm-up
    r0 = pool.stats()["rays"]
    t0 = time.perf_counter()
    recs = serve(pool, arrivals)
    wall = time.perf_counter() - t0
    rays = pool.stats()["rays"] - r0
    lat = np.array([r["latency"] for r in recs])
    samples = sum(j.width * j.height * j.frames for _, j in arrivals)
    pool.close()
    return {"metric": METRIC, "value": rays / wall / 1e6, "unit": "Mrays/s",
            "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)),
            "mean_latency_s": float(lat.mean()), "jobs": len(recs),
            "arrival_span_s": arrivals[-1][0], "wall_seconds": wall, "rays": rays,
            "samples": samples,
            "offered_samples_per_s": samples / max(arrivals[-1][0], 1e-9),
            "config": {**SERVE, "jobs": n, "capacity_samples": 1 << 21,
                       "camera": "uniform on a sphere of radius 2 around the box centre",
                       "admission": "first come first served by free HBM"},
            "note": "latency on the host clock (arrival -> end of the finishing iteration); "
                    "Mrays/s = rays traced / wall time of the serving window; the offered "
                    "load exceeds the device's throughput, so latency includes queueing"}


# ---- learned guiding --------------------------------------------------------
C1 = {"Samples": 2, "MaxDepth": 5, "NextEventEstimation": 1, "RussianRouletteStart": 3,
      "DirectLightMIS": 0}
# GuideBounceAmount 2: both guiders guide the first two bounces, where the
# indirect light they learn is; later bounces carry little of the image and
# their guiding costs more than it returns (shielded scene, four seeds)
LEARNED = {"LearnedGuiding": 1, "LearnedWarmupFrames": 16, "LearnedTrainSteps": 1,
           "LearnedSamples": 65536, "LearnedWarmupOctree": 0, "OctreeLevel": 10,
           "MinRayBinLevel": 5, "BinRayCount": 512, "GuideBounceAmount": 2}
LEARNED_FLOATS = {"LearnedRate": 1e-2, "LearnedWeightMax": 5.0, "BXDF-GuideMISRatio": 0.5,
                  "RFieldFilterAlpha": 0.6}


def _frame_ms(t, torch, frames=20):
    stream = torch.cuda.ExternalStream(t.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(frames):
        t.render_frame()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / frames


def run_learned(args, m, system, torch) -> dict:
    """The learned-guiding comparison on the config Cornell scene and on its
    shielded-light variant (light reaching the room only by way of the
    ceiling), where guiding has indirect light to find."""
    out = _run_learned_scene(args, m, system, torch, shielded=False)
    out["shielded_light"] = _run_learned_scene(args, m, system, torch, shielded=True)
    return out


def _run_learned_scene(args, m, system, torch, shielded: bool) -> dict:
    """Learned guiding on the 8k-triangle Cornell scene (128x128, 4 spp per
    frame, depth 5): plain path tracing, SVO path guiding and learned guiding
    (MLP vMF mixture trained online on the tensor cores; its first 16 frames
    sampled by the BxDF alone, or by the octree guider for "_octree") get
    the same device-time budget from a cold start and are scored by mean
    squared error against a 16384-spp plain render, less that render's own
    variance."""
    scene = m.scenes.cornell(seed=1, shielded=shielded)
    g = m.GPUScene(system, scene)
    g.construct_accelerators()

    def make(kind, seed):
        plain = kind in ("plain", "plain_nee")
        t = m.PathTracer(system, g) if plain else m.WFPGTracer(system, g)
        # NEE off for every estimator, as the reference's own WFPG
        # configurations run (WorkingDir/tConf_veach_product.json): with
        # NEE, next to the ceiling light NEE throws fireflies that dominate
        # every MSE (plain_nee: NEE as configured), and with NEE and MIS the
        # guided estimators are biased (the NEE weight uses the BxDF pdf,
        # the guided path ray the mixture pdf, WFPGTracerKC.cuh:338-347)
        opts = dict(C1, Seed=seed, NextEventEstimation=1 if kind == "plain_nee" else 0)
        if plain:
            t.set_options(opts)
            return t
        if kind == "wfpg_bxdf":
            # the same tracer with its network never taking over: the BxDF
            # samples every frame (the method without the network)
            opts.update(LEARNED, LearnedWarmupFrames=1 << 30)
            t.set_options(opts)
            t.set_options(LEARNED_FLOATS)
            return t
        learned = kind.startswith("learned")
        if kind != "plain":
            opts.update({k: v for k, v in LEARNED.items()
                         if learned or not k.startswith("Learned")})
            if learned:
                opts["LearnedTrainSteps"] = int(kind.split("_")[1])
                opts["LearnedWarmupOctree"] = 1 if kind.endswith("_octree") else 0
        t.set_options(opts)
        if kind != "plain":
            t.set_options({k: v for k, v in LEARNED_FLOATS.items()
                           if learned or not k.startswith("Learned")})
        return t

    # the converged render: NEE with MIS (the same expectation as every
    # estimator here, without the fireflies NEE alone throws next to the light)
    def make_ref(seed):
        t = m.PathTracer(system, g)
        t.set_options(dict(C1, Seed=seed, DirectLightMIS=1))
        return t
    ref_img, ref_var, ref_rvar = _reference(lambda half: make_ref(4242 + half),
                                            args.learned_reference_spp // 4)
    out = {"budget_ms": args.learned_budget_ms, "reference_spp": args.learned_reference_spp,
           "reference_variance": ref_var}
    kinds = (("plain", 11), ("wfpg_bxdf", 16), ("svo", 12), ("learned_1", 13), ("learned_4", 14),
             ("learned_1_octree", 15), ("plain_nee", 17))
    if args.learned_kinds:
        kinds = tuple(k for k in kinds if k[0] in args.learned_kinds.split(","))
    for kind, seed in kinds:
        probe = make(kind, seed + 100)
        for _ in range(24):           # past the warm-up: the frame time the budget meets
            probe.render_frame()
        ms = _frame_ms(probe, torch)
        probe.close()
        t = make(kind, seed)
        img, frames, used = _budget_image(t, args.learned_budget_ms, ms, torch)
        raw = float(np.mean((img - ref_img) ** 2))
        entry = {"ms_per_frame": ms, "frames": frames, "spp": 4 * frames, "device_ms": used,
                 "mse": raw - ref_var, "mse_raw": raw,
                 "rel_mse": _rel_mse(img, ref_img) - ref_rvar,
                 "clamped_mse": _clamped_mse(img, ref_img)}
        if kind.startswith("learned"):
            entry["held_out_loss_last_frame"] = t.learned_loss()
            entry["train_steps_per_frame"] = int(kind.split("_")[1])
            entry["warm_up_sampler"] = "octree" if kind.endswith("_octree") else "BxDF"
        t.close()
        out[kind] = entry
    if all(k in out for k in ("plain", "wfpg_bxdf", "svo", "learned_1", "learned_4",
                              "learned_1_octree")):
        best = min(("learned_1", "learned_4", "learned_1_octree"), key=lambda k: out[k]["mse"])
        out["learned"] = dict(out[best], variant=best)
        out["learned_over_plain"] = out["learned"]["mse"] / out["plain"]["mse"]
        out["learned_over_wfpg_bxdf"] = out["learned"]["mse"] / out["wfpg_bxdf"]["mse"]
        out["learned_over_svo"] = out["learned"]["mse"] / out["svo"]["mse"]
        # the same ratios on the relative MSE (the learned variant with the
        # lowest one), which rare high-energy paths move less
        best_rel = min(("learned_1", "learned_4", "learned_1_octree"),
                       key=lambda k: out[k]["rel_mse"])
        out["rel_mse_learned_variant"] = best_rel
        out["learned_over_plain_rel"] = out[best_rel]["rel_mse"] / out["plain"]["rel_mse"]
        out["learned_over_wfpg_bxdf_rel"] = (out[best_rel]["rel_mse"]
                                             / out["wfpg_bxdf"]["rel_mse"])
        # per-sample efficiency (MSE x spp; lower is better), which the frame
        # cost then trades against
        out["mse_x_spp"] = {k: out[k]["mse"] * out[k]["spp"]
                            for k in ("plain", "wfpg_bxdf", "svo", "learned_1", "learned_4",
                                      "learned_1_octree", "plain_nee") if k in out}
    out["config"] = {"scene": ("Cornell box (seed 1) with the light facing the ceiling over an "
                               "opaque panel" if shielded else
                               "Cornell box with a ceiling-wide light (seed 1)")
                     + ", 128x128, 4 spp per frame, depth 5, NEE off (plain_nee: the plain "
                       "tracer with NEE); reference: plain, NEE with MIS",
                     **LEARNED, **LEARNED_FLOATS,
                     "network": "80-64-64-64-40 ReLU MLP, 8 vMF lobes, BF16 weights and "
                                "activations, FP32 accumulation on tcgen05 tensor cores"}
    return out


def _oracle_setup(scene):
    """Scene arrays as the hot path consumes them, built by the oracle alone."""
    from oracle import oracle as o
    return o.OracleScene.from_scene(scene)


def _camera16(scene):
    """Pinhole frame (GPUCameraPinhole.cuh:135-162) computed in float32."""
    f = np.float32
    c = scene.camera
    pos = np.array(c["position"], f)
    gz = np.array(c["gaze"], f)
    up = np.array(c["up"], f)
    near = f(c["near_far"][0])
    wh = f(np.tan(f(c["fov"][0]) * f(0.5))) * near
    hh = f(np.tan(f(c["fov"][1]) * f(0.5))) * near

    def nrm(v):
        return (v * (f(1) / np.sqrt(np.dot(v, v), dtype=f))).astype(f)

    gd = gz - pos
    right = nrm(np.cross(gd, up).astype(f))
    up = nrm(np.cross(right, gd).astype(f))
    gd = nrm(np.cross(up, right).astype(f))
    bl = ((pos - right * wh) - up * hh) + gd * near
    return np.concatenate([pos, bl, right, up, [wh * 2, hh * 2],
                           np.array(c["near_far"], f)]).astype(f)


# The CPU legs (cpu_baseline of the GPU arm and the --impl reference arm)
# time the same row-stratified sample of the full 1920x1080 frame: step i
# renders every CPU_ROW_STRIDE-th image row starting at row i mod
# CPU_ROW_STRIDE, so CPU_ROW_STRIDE consecutive steps cover the whole frame
# once and every step sees the top, middle and bottom of the image alike.
CPU_ROW_STRIDE = 4


def _load_scenes():
    """The seeded scene generator, loaded from its file on its own: the CPU
    legs must not import the package (which maps libmrb200.so)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("mrb_scenes_standalone",
                                                  ROOT / "meturay_b200" / "scenes.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod  # dataclasses resolve their module by name
    spec.loader.exec_module(mod)
    return mod


def cpu_leg(scene, os_, step: int, threads: int) -> dict:
    """One CPU step: the rows r = step mod CPU_ROW_STRIDE (mod CPU_ROW_STRIDE)
    of the frame, at the frame index of the step (1 spp, depth 8, NEE)."""
    cf = _camera16(scene)
    t0 = time.perf_counter()
    _, rays = os_.render(cf, scene.width, scene.height, 1, 8, 3, True, 1, frame=step,
                         threads=threads, rows=(step % CPU_ROW_STRIDE, scene.height),
                         row_step=CPU_ROW_STRIDE)
    dt = time.perf_counter() - t0
    return {"rays": rays, "seconds": dt}


def cpu_sample_text(scene, steps: int, cores: int) -> str:
    return (f"{steps} steps; step i renders every {CPU_ROW_STRIDE}th row of the "
            f"{scene.width}x{scene.height} clusters-1M frame from row i mod {CPU_ROW_STRIDE} "
            f"({scene.height // CPU_ROW_STRIDE} rows, 1 spp, depth 8), {cores} threads")


def run_reference(args) -> dict:
    scenes = _load_scenes()
    cores = os.cpu_count() or 1
    scene = scenes.clusters(seed=1)
    os_ = _oracle_setup(scene)
    for w in range(args.warmup):
        cpu_leg(scene, os_, w, cores)
    total_rays, total_s = 0, 0.0
    for i in range(args.steps):
        r = cpu_leg(scene, os_, i, cores)
        total_rays += r["rays"]
        total_s += r["seconds"]
    value = total_rays / total_s / 1e6
    return {
        "metric": METRIC, "value": value, "unit": "Mrays/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_s * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded clusters-1M scene)",
        "config": run_config(args.gpus),
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": cores, "kind": "port",
                         "sample": cpu_sample_text(scene, args.steps, cores)},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def run_config(world: int) -> dict:
    """The workload of the line; both arms report the same one."""
    return dict(WORKLOAD, parallelism=f"replicas{world}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--traversal", type=int, default=1, choices=[0, 1],
                    help="1: 8-wide quantised BVH (default), 0: binary LBVH nodes")
    ap.add_argument("--no-guided", dest="guided", action="store_false",
                    help="skip the WFPG (SVO path guiding) run")
    ap.add_argument("--mse-budget-ms", type=float, default=2000.0,
                    help="equal-time MSE budget per tracer (0 skips the comparison)")
    ap.add_argument("--mse-reference-spp", type=int, default=2048)
    ap.add_argument("--no-pool", dest="pool", action="store_false",
                    help="skip the wavefront-pool batching and serving runs")
    ap.add_argument("--serve-jobs", type=int, default=64,
                    help="jobs in the serving run (Poisson arrivals at 200/s)")
    ap.add_argument("--pool-block", type=int, default=0)
    ap.add_argument("--pool-stack", type=int, default=128,
                    help="traversal stack of the pool: 64 or 128 (sorted order) or 0 (octant order)")
    ap.add_argument("--wide-order", default="auto",
                    choices=["auto", "sorted", "octant", "sorted_refill", "octant_refill"],
                    help="8-wide traversal kernel of the headline frame (auto: timed per depth)")
    ap.add_argument("--wide-collapse", type=int, default=2, choices=[0, 1, 2],
                    help="8-wide node children: 0 largest area first, 1 the surface-area plan, "
                         "2 the one the probe rays read less of")
    ap.add_argument("--no-closed", dest="closed", action="store_false",
                    help="skip the bounce-heavy Cornell 1080p 4 spp entry")
    ap.add_argument("--no-learned", dest="learned", action="store_false",
                    help="skip the learned-guiding equal-time MSE comparison")
    ap.add_argument("--learned-budget-ms", type=float, default=1000.0)
    ap.add_argument("--learned-reference-spp", type=int, default=16384)
    ap.add_argument("--learned-kinds", default="",
                    help="comma list of plain,wfpg_bxdf,svo,learned_1,learned_4,"
                         "learned_1_octree (default all)")
    ap.add_argument("--only", choices=["all", "guided", "learned", "closed"], default="all",
                    help="guided: only the WFPG timing (for profiling a small case); "
                         "learned: only the learned-guiding comparison; closed: only the "
                         "closed-scene entry")
    ap.add_argument("--res", default="1920x1080",
                    help="image size WxH (the workload is 1920x1080; smaller for profiling)")
    args = ap.parse_args()
    args.res = tuple(int(v) for v in args.res.lower().split("x"))
    if args.warmup < 3:
        args.warmup = 3

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)))
        return

    dist = None
    if world > 1:
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    out = run_ours(args, rank, world, dist)
    if out is not None and not args.no_cpu_baseline and args.only == "all":
        # the reference arm's sample: 2 x CPU_ROW_STRIDE steps = the whole
        # frame twice (about 5-10 s on the host's cores)
        scene = _load_scenes().clusters(seed=1)
        os_ = _oracle_setup(scene)
        cores = os.cpu_count() or 1
        cpu_leg(scene, os_, 0, cores)  # warm-up
        from oracle import oracle as o
        o.trace_counters(reset=True)
        steps = 2 * CPU_ROW_STRIDE
        tot_r, tot_s = 0, 0.0
        for i in range(steps):
            r = cpu_leg(scene, os_, i, cores)
            tot_r += r["rays"]
            tot_s += r["seconds"]
        visits, tris = o.trace_counters()
        out["cpu_baseline"] = {"value": tot_r / tot_s / 1e6, "unit": "Mrays/s",
                               "cores": cores, "kind": "port",
                               "sample": cpu_sample_text(scene, steps, cores)
                               + f", {tot_s:.1f} s"}
        # the same frame's work counted independently of the GPU kernels: the
        # oracle's traversal of the reference's binary LBVH over the CPU
        # sample's rays, scaled to the GPU frame's ray count
        roof = out["roofline"]
        vpr, tpr = visits / max(tot_r, 1), tris / max(tot_r, 1)
        nr = roof["rays_per_frame"]
        tb = trace_bytes(nr, vpr * nr, tpr * nr, 0)
        ach = tb / (roof["trace_ms_per_frame"] / 1e3) / 1e9
        roof["reference_tree"] = {
            "source": "oracle traversal of the binary LBVH (the reference's tree and "
                      "traversal order) over the cpu_baseline sample's rays",
            "node_visits_per_ray": vpr, "tri_tests_per_ray": tpr,
            "algorithmic_bytes_per_frame": tb, "achieved": ach, "frac": ach / roof["peak"],
            "note": "the reference tree's work done in the 8-wide kernels' time; above 1.0 "
                    "where the 8-wide layout visits fewer, smaller nodes than the binary "
                    "tree would stream"}
    if out is not None:
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
