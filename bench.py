#!/usr/bin/env python
"""Training-step throughput of the QSDVR render path on B200 (rays/s, fwd+bwd).

Workload (default ``plain256``): 256^3 quadric grid + [(257)^3, 32] appearance grid, fp32,
100 seeded views at 800x800 (focal 1111.1 px, upper hemisphere at radius 4.03), 65536
random rays per step, 256 samples/ray over t in [2, 6] (interval 4/256).  Targets are
rendered from a seeded procedural ground-truth scene.  One step = one fused forward + MSE +
backward launch over the batch, its gradients accumulated into fp32 buffers zeroed before
the timed region; zeroing, the fused Adam step and a full training step are timed beside it
(``step_parts``).  Inputs (2.7 GB of grids) are far larger than L2, so no flush is needed
between steps.  The line also carries ``proposal``: training with the proposal network's
samples against the uniform march, rays/s and held-out PSNR of each.

``--impl reference`` times the reference's own CPU path (its pure-torch renderer with the
per-ray compositing loop, restated to run on the host) on a bounded sample of the same
workload and prints the same JSON line with "impl": "reference".

Launch: python bench.py [--gpus N --steps K --warmup W]; for N > 1 under torchrun (one
replica per GPU, each with its own batches: weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: grid R, rays/step, views, image size, focal, camera radius, interval, storage
    "plain256": dict(R=256, rays=65536, views=100, size=800, focal=1111.1, radius=4.03, interval=4.0 / 256,
                     storage="f32"),
    "bf16_256": dict(R=256, rays=65536, views=100, size=800, focal=1111.1, radius=4.03, interval=4.0 / 256,
                     storage="bf16"),
    # the precision form with the appearance gradient accumulated in bf16 (SDF gradient fp32)
    "bf16g_256": dict(R=256, rays=65536, views=100, size=800, focal=1111.1, radius=4.03, interval=4.0 / 256,
                      storage="bf16", grad="bf16"),
    "plain128": dict(R=128, rays=8192, views=100, size=800, focal=1111.1, radius=4.03, interval=4.0 / 256,
                     storage="f32"),
    # SH degree 3 (64-channel rows, fixed mode): the configs' appearance model
    "sh3_256": dict(R=256, rays=65536, views=100, size=800, focal=1111.1, radius=4.03, interval=4.0 / 256,
                    storage="f32", sh=3),
    "sh3_bf16_256": dict(R=256, rays=65536, views=100, size=800, focal=1111.1, radius=4.03, interval=4.0 / 256,
                         storage="bf16", sh=3),
    "sh3_128": dict(R=128, rays=8192, views=100, size=800, focal=1111.1, radius=4.03, interval=4.0 / 256,
                    storage="f32", sh=3),
    # learned proposal form: full-frame renders of a trained 384^3 BF16 SH3 model, 64 coarse MLP
    # points + 32 fine samples per ray against the 512-sample uniform march
    # the proposal network's kernels at the training batch: coarse MLP inference (64 points per
    # ray) against the tensor roofline, beside the sampler, MLP training and the renders
    "mlp256": dict(R=256, rays=65536, views=20, size=800, focal=1111.1, radius=4.03, interval=4.0 / 256,
                   storage="f32", online_steps=200),
    "proposal384": dict(R=384, rays=65536, views=200, size=800, focal=1111.1, radius=4.03, interval=4.0 / 512,
                        storage="bf16", sh=3, train_steps=200, heldout=4),
    # training comparison at 512 samples/ray (the learned proposal form's uniform march) on the
    # 256^3 scene: proposal path against the uniform march, rays/s and held-out PSNR
    "train512": dict(R=256, rays=65536, views=100, size=800, focal=1111.1, radius=4.03, interval=4.0 / 512,
                     storage="f32"),
    # small cases of the proposal kernels and of the frame forwards, sized for profiler captures
    # (a few GB on the device): the same kernels as mlp256 and proposal384 on a 128^3 grid
    "mlp128": dict(R=128, rays=65536, views=4, size=800, focal=1111.1, radius=4.03, interval=4.0 / 256,
                   storage="f32", online_steps=50),
    "proposal128": dict(R=128, rays=16384, views=20, size=400, focal=555.55, radius=4.03, interval=4.0 / 512,
                        storage="bf16", sh=3, train_steps=50, heldout=1),
    # the reference's small CPU-runnable case: a 64^3 noisy sphere, one 100x100 view at radius 4
    # (focal 138.9), 64 samples/ray, every pixel's ray, MSE against a seeded U(0,1) image
    "config1": dict(R=64, rays=10000, views=1, size=100, focal=138.9, radius=4.0, interval=4.0 / 64,
                    storage="f32", scene="sphere"),
}
CONFIG1_CAMERA = (0.0, -4.0, 0.0)  # radius 4, looking at the origin
PROPOSAL_STEPS = 300  # training steps per method in the default line's proposal comparison


def byte_terms(storage: str, sh: int, grad: str = "f32") -> tuple[int, int, int]:
    """Algorithmic bytes of the train kernel: (per render sample, per sample whose SDF sample
    has a gradient, per active sample).  Every sample reads its two quadric cells (SDF sample
    i+1 and the render sample's cell, 2 x 32 B).  The SDF sample's cell gradient is
    read-modify-written (64 B) when it is not zero, i.e. when alpha > 0 on either interval the
    sample bounds.  An active sample, one with alpha > 0, also read-modify-writes its render
    cell's normal gradient (64 B), gathers its 8 corner rows once (8 C b; the backward rereads
    them from the warp's L2 stash) and read-modify-writes its 8 gradient rows in L2
    (2 x 8 C g).  An inactive sample's colour terms are all zero: its rows are neither
    gathered nor sent.  C channels, b storage bytes, g gradient bytes."""
    c = 32 if sh == 2 else 64
    b = 4 if storage == "f32" else 2
    g = 4 if grad == "f32" else 2
    return 64, 64, 64 + 8 * c * b + 2 * 8 * c * g


def bytes_per_sample(storage: str, sh: int, grad: str = "f32", active: float = 1.0,
                     sdf_grad: float | None = None) -> float:
    """Algorithmic bytes per render sample when a fraction ``active`` of them is active and a
    fraction ``sdf_grad`` (default: ``active``) sends an SDF-cell gradient."""
    every, per_sdf, per_active = byte_terms(storage, sh, grad)
    return every + (active if sdf_grad is None else sdf_grad) * per_sdf + active * per_active


BYTES_PER_RAY = 64  # origin + dir in, target in, colour out, RayInfo
K_LOGISTIC = 5.0
METRIC = "train rays/s fwd+bwd @256^3 grid (256 samples/ray, 65536-ray batches)"


def max_over_ranks(values, device, ws):
    """Every rank's timings replaced by their maximum over the ranks (the job is as slow as
    its slowest replica)."""
    t = torch.tensor(values, dtype=torch.float64, device=device)
    if ws > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return t.tolist()


def job_throughput(rays_per_step: int, steps: int, ws: int, max_ms: float) -> float:
    """Whole-job rays/s: every replica's rays over the slowest replica's time."""
    return rays_per_step * steps * ws / (max_ms / 1e3)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 20 ms during the timed region."""

    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "20"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self, begin: bool):
        """Record the wall-clock bounds of a timed region."""
        if begin:
            self.t0 = time.time()
        else:
            self.t1 = time.time()

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        """Samples that arrived inside the timed window (plus one sampling period on each
        side; the nearest two if the window is shorter than the sampling period)."""
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        parsed = []
        for t, ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                parsed.append((t, float(parts[1]), float(parts[2]), parts[4:8]))
            except ValueError:
                continue
        t0, t1 = getattr(self, "t0", 0.0), getattr(self, "t1", float("inf"))
        inside = [q for q in parsed if t0 - 0.05 <= q[0] <= t1 + 0.05]
        if len(inside) < 2 and parsed:
            mid = 0.5 * (t0 + min(t1, parsed[-1][0]))
            inside = sorted(parsed, key=lambda q: abs(q[0] - mid))[:2]
        sm = [q[1] for q in inside]
        reasons = set()
        for q in inside:
            for nm, v in zip(names, q[3]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": inside[0][2] if inside else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic_per_sample(storage: str):
    """DRAM bytes per render sample of the train kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "fused_train_dram.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith(f"dram_bytes_per_render_sample_{storage}:"):
                    return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


# ----------------------------------------------------------------------------- setup

def build_scene(cfg, device, seed):
    """Ground-truth scene (targets), trained model, and the ray tables of all views."""
    from qsdvr_b200 import fused, scenes
    from qsdvr_b200.camera import Camera

    R = cfg["R"]
    if cfg.get("scene") == "sphere":  # config1: the model is the noisy sphere; targets are U(0,1)
        cam = Camera(scenes.look_at(CONFIG1_CAMERA, cfg["size"], cfg["size"], cfg["focal"], 2.0, 6.0),
                     cfg["interval"], R, device=device)
        cam.GenerateRayPoints(torch.ones(cfg["size"] * cfg["size"], dtype=torch.bool))
        sdf = fused.pad_grid7(scenes.sphere_grid(R, 0.5, 0.01, seed=seed, device=device).reshape(-1, 7))
        data = scenes.appearance(R, seed=seed, device=device)
        return dict(gt=None, model=(sdf, data), rays=cam.rayList, origin=cam.originList, dir=cam.dirList)
    gt_sdf = fused.pad_grid7(scenes.procedural_grid(R, seed=seed, device=device).reshape(-1, 7))
    sh = cfg.get("sh", 2)
    gt_data = scenes.appearance(R, seed=seed, device=device, procedural=True, sh_degree=sh)
    sdf = fused.pad_grid7(scenes.sphere_grid(R, 0.5, 0.01, seed=seed, device=device).reshape(-1, 7))
    data = scenes.appearance(R, seed=seed + 1, device=device, sh_degree=sh)
    cams = scenes.hemisphere_cameras(cfg["views"], cfg["radius"], cfg["size"], cfg["size"], cfg["focal"], 2.0, 6.0,
                                     seed=seed)
    rays, origin, direction = [], [], []
    mask = torch.ones(cfg["size"] * cfg["size"], dtype=torch.bool)
    for a in cams:
        c = Camera(a, cfg["interval"], R, device=device)
        c.GenerateRayPoints(mask)
        rays.append(c.rayList)
        origin.append(c.originList)
        direction.append(c.dirList)
    return dict(gt=(gt_sdf, gt_data), model=(sdf, data), rays=torch.cat(rays), origin=torch.cat(origin),
                dir=torch.cat(direction))


def make_batches(scene, cfg, count, device, seed):
    from qsdvr_b200 import fused

    if scene["gt"] is None:  # config1: every pixel's ray in pixel order, targets U(0,1) (seed 0)
        target = torch.rand((scene["rays"].shape[0], 3), generator=torch.Generator().manual_seed(0)).to(device)
        return [dict(rays=scene["rays"], origin=scene["origin"], dir=scene["dir"], target=target)] * count
    gen = torch.Generator(device=device).manual_seed(seed)
    total = scene["rays"].shape[0]
    out = []
    for _ in range(count):
        idx = torch.randint(0, total, (cfg["rays"],), generator=gen, device=device)
        b = dict(rays=scene["rays"][idx].contiguous(), origin=scene["origin"][idx].contiguous(),
                 dir=scene["dir"][idx].contiguous())
        gs, gd = scene["gt"]
        b["target"] = fused.render_forward(b["rays"], b["origin"], b["dir"], gs, gd, cfg["R"], cfg["interval"],
                                           K_LOGISTIC, "fixed")
        out.append(b)
    return out


def samples_of(batch):
    c = batch["rays"][:, 0].long()
    return int(torch.clamp(c - 1, min=0).sum())


def active_samples_of(batch, sdf_k, data_k, R, interval, mode, transmittance):
    """(samples with alpha > 0, samples whose SDF sample has a gradient: alpha > 0 on its own
    interval or on the next one of the same ray) under the model, counted outside any timed
    region with one forward of the library and its per-sample alpha output (the ray records
    given packed render offsets; the fused kernels read only sdf_count besides)."""
    from qsdvr_b200 import fused

    rays = batch["rays"].clone()
    cnt = torch.clamp(rays[:, 0].long() - 1, min=0)
    rays[:, 2] = cnt.to(torch.int32)
    off = torch.cumsum(cnt, 0) - cnt
    rays[:, 3] = off.to(torch.int32)
    alpha = torch.zeros(int(cnt.sum()), dtype=torch.float32, device=rays.device)
    fused.render_forward(rays, batch["origin"], batch["dir"], sdf_k, data_k, R, interval, K_LOGISTIC, mode,
                         transmittance, sample_alpha=alpha)
    act = alpha > 0
    nxt = torch.zeros_like(act)
    nxt[:-1] = act[1:]
    last = (off + cnt - 1)[cnt > 0]  # a ray's last sample has no next interval in the ray
    nxt[last] = False
    return int(act.sum()), int((act | nxt).sum())


# ----------------------------------------------------------------------------- timing

def time_device(step, steps, warmup, stream, clock=None, on_start=None):
    """Warm-up, then K steps between two events; also returns per-step kernel events.
    ``on_start(start_event)`` lets other streams of the step wait for the region's start."""
    for i in range(warmup):
        step(i, None)
    torch.cuda.synchronize()
    if clock is not None:
        clock.mark(True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("timed")
    start.record(stream)
    if on_start is not None:
        on_start(start)
    for i in range(steps):
        step(i, ev[i])
    stop.record(stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    if clock is not None:
        clock.mark(False)
    total_ms = start.elapsed_time(stop)
    kern_ms = [a.elapsed_time(b) for a, b in ev]
    return total_ms, kern_ms


def run_ours(args, cfg, device, ws, rank):
    from qsdvr_b200 import fused

    R = cfg["R"]
    storage = cfg["storage"]
    scene = build_scene(cfg, device, seed=0)
    batches = make_batches(scene, cfg, 8, device, seed=1000 + rank)
    sdf, data = scene["model"]
    transmittance = "log" if storage == "bf16" else "product"
    mode = "compat" if cfg.get("sh", 2) == 2 else "fixed"
    if storage == "bf16":
        sdf_k, data_k = fused.sdf_cells_bf16(sdf), data.to(torch.bfloat16)
    else:
        sdf_k, data_k = sdf, data
    sg = torch.zeros(sdf.shape, dtype=torch.float32, device=device)
    grad_dtype = torch.bfloat16 if cfg.get("grad", "f32") == "bf16" else torch.float32
    dg = torch.zeros(data.shape, dtype=grad_dtype, device=device)
    loss = torch.zeros(1, dtype=torch.float32, device=device)
    color = torch.empty((cfg["rays"], 3), dtype=torch.float32, device=device)
    stream = torch.cuda.current_stream(device)

    # gradients accumulate over the steps into buffers zeroed once before timing (the
    # scatter's work does not depend on what the buffers hold); zeroing and the optimizer
    # step are timed separately below, and a full training step beside them
    # each step takes its rays in the Morton order of their midpoints (the library's counting
    # sort inside the timed step; the kernel events bracket the train launch alone)
    def step(i, ev):
        b = batches[i % len(batches)]
        loss.zero_()
        order = fused.ray_order(b["rays"], b["origin"], b["dir"], cfg["interval"])
        if ev is not None:
            ev[0].record(stream)
        fused.render_train(b["target"], b["rays"], b["origin"], b["dir"], sdf_k, data_k, R, cfg["interval"],
                           K_LOGISTIC, sg, dg, mode, transmittance, loss=loss, color=color, order=order,
                           merge=args.merge)
        if ev is not None:
            ev[1].record(stream)

    if ws > 1:
        torch.distributed.barrier()
    with ClockSampler(device.index) as clk:
        time.sleep(0.3)  # nvidia-smi needs a moment before its first sample
        total_ms, kern_ms = time_device(step, args.steps, args.warmup, stream, clk)
    if ws > 1:
        torch.distributed.barrier()
    # samples with a non-zero appearance gradient under the model the timed region used (the
    # full-step timing below updates the model)
    counts = [active_samples_of(b, sdf_k, data_k, R, cfg["interval"], mode, transmittance) for b in batches]
    all_samples = max(1, sum(samples_of(b) for b in batches))
    active_frac = sum(c[0] for c in counts) / all_samples
    sdf_grad_frac = sum(c[1] for c in counts) / all_samples
    # ---- e2e through the public API with host buffers (pinned), copies inside the region
    host = []
    for b in batches:
        host.append({k: v.cpu().pin_memory() for k, v in b.items()})
    # two device input buffers: step i's batch is copied on a copy stream while step i-1's
    # kernel runs (the copy waits until step i-2 has released the buffer)
    dev_in = [{k: torch.empty_like(v) for k, v in batches[0].items()} for _ in range(2)]
    copy_stream = torch.cuda.Stream(device)
    copied = [torch.cuda.Event() for _ in range(2)]
    released = [torch.cuda.Event() for _ in range(2)]
    for e in released:
        e.record(stream)
    loss_host = torch.zeros(1, dtype=torch.float32).pin_memory()
    h2d = sum(v.numel() * v.element_size() for v in host[0].values())

    def e2e_step(i, ev):
        hb, buf = host[i % len(host)], dev_in[i % 2]
        with torch.cuda.stream(copy_stream):
            copy_stream.wait_event(released[i % 2])
            for k, v in hb.items():
                buf[k].copy_(v, non_blocking=True)
            copied[i % 2].record(copy_stream)
        loss.zero_()
        stream.wait_event(copied[i % 2])
        if ev is not None:
            ev[0].record(stream)
        order = fused.ray_order(buf["rays"], buf["origin"], buf["dir"], cfg["interval"])
        fused.render_train(buf["target"], buf["rays"], buf["origin"], buf["dir"], sdf_k, data_k, R,
                           cfg["interval"], K_LOGISTIC, sg, dg, mode, transmittance, loss=loss, color=color,
                           order=order, merge=args.merge)
        if ev is not None:
            ev[1].record(stream)
        released[i % 2].record(stream)
        loss_host.copy_(loss, non_blocking=True)

    if ws > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    e2e_ms, _ = time_device(e2e_step, args.steps, args.warmup, stream, on_start=copy_stream.wait_event)
    wall_e2e = time.perf_counter() - t0
    step_parts = full_step_parts(args, cfg, batches, sdf, data, sdf_k, data_k, sg, dg, mode, transmittance, loss,
                                 color, stream)
    # ---- aggregate over ranks (max time)
    total_ms, e2e_ms, kern_avg = max_over_ranks([total_ms, e2e_ms, sum(kern_ms) / len(kern_ms)], device, ws)
    value = job_throughput(cfg["rays"], args.steps, ws, total_ms)
    e2e_value = job_throughput(cfg["rays"], args.steps, ws, e2e_ms)
    # ---- roofline of the train kernel
    samples = [samples_of(b) for b in batches]
    mean_samples = sum(samples) / len(samples)
    bps = bytes_per_sample(storage, cfg.get("sh", 2), cfg.get("grad", "f32"), active_frac, sdf_grad_frac)
    alg_bytes = mean_samples * bps + cfg["rays"] * BYTES_PER_RAY
    achieved = alg_bytes / (kern_avg / 1e3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    tps = profiled_traffic_per_sample(storage + ("_sh3" if cfg.get("sh", 2) == 3 else "")
                                      + ("_grad_bf16" if cfg.get("grad", "f32") == "bf16" else ""))
    # the committed DRAM capture covers the 256^3 workloads only
    traffic = None if tps is None or R != 256 else tps * mean_samples
    out = {
        "metric": METRIC, "value": round(value, 1), "unit": "rays/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if storage == "f32" else ("bf16 storage, f32 math" + (", bf16 appearance gradient"
                                                                          if cfg.get("grad") == "bf16" else "")),
        "data": "synthetic (seeded procedural scene, random-init sphere model)",
        "config": {"workload": f"{args.workload}: R={R}^3 quadric + ({R + 1})^3x{32 if cfg.get('sh', 2) == 2 else 64} "
                               f"appearance grid, {storage}, "
                               + (f"every pixel's ray of one {cfg['size']}^2 view, " if cfg.get("scene") == "sphere"
                                  else f"{cfg['rays']} random rays/step from {cfg['views']} views at {cfg['size']}^2, ")
                               + f"interval {cfg['interval']:.6g} ({round(4.0 / cfg['interval'])} samples/ray), SH degree {cfg.get('sh', 2)}, "
                               f"{mode} mode, k={K_LOGISTIC}"
                               + (", same-cell merged appearance scatter" if args.merge else ""),
                   "global_batch": cfg["rays"] * ws, "samples_per_step": round(mean_samples),
                   "step": "the ray order (the library's counting sort of the rays' midpoints on a 32^3 "
                           "Morton lattice: bucket, scan and scatter kernels), then one fused forward/MSE/"
                           "backward launch; gradients accumulated into buffers zeroed before the timed region "
                           "(zeroing, optimizer and full step in step_parts)",
                   "l2": "inputs larger than L2 (grids 2.7 GB), no flush", "parallelism": f"replicas x{ws}"},
        "e2e": {"value": round(e2e_value, 1), "unit": "rays/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 4,
                "wall_s": round(wall_e2e, 3)},
        "gpu_launches": 4 * args.steps,  # qsdvr_ray_order's 3 kernels + the train kernel per step
        "step_parts": step_parts,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": None if traffic is None else round(traffic),
                     "kernel": "render_kernel<train>", "kernel_ms": round(kern_avg, 4),
                     "algorithmic_bytes": round(alg_bytes), "bytes_per_sample": round(bps, 1),
                     "active_sample_fraction": round(active_frac, 4),
                     "sdf_grad_sample_fraction": round(sdf_grad_frac, 4),
                     "peak_kind": peak_kind},
        "clocks": clk.summary(),
    }
    # the reference's CPU path is SH degree 2; config1's full case is timed by --impl reference
    if ws == 1 and not args.no_cpu_baseline and cfg.get("sh", 2) == 2 and cfg.get("scene") != "sphere":
        out["cpu_baseline"] = cpu_baseline(scene, batches[0], cfg, args.cpu_rays)
    if ws == 1 and args.workload == "plain256" and not args.no_proposal:
        del scene, batches
        torch.cuda.empty_cache()
        out["proposal"] = proposal_comparison(PROPOSAL_STEPS, args.proposal_warmup)
        # the same comparison on bf16 storage (both methods; the learned proposal form's precision)
        out["proposal_bf16"] = proposal_comparison(PROPOSAL_STEPS, args.proposal_warmup, storage="bf16")
    return out


def full_step_parts(args, cfg, batches, sdf, data, sdf_k, data_k, sg, dg, mode, transmittance, loss, color, stream):
    """The pieces of a full training step beside the timed forward + backward: zeroing the
    fp32 gradient buffers, the fused Adam step (fp32 masters, bf16 copies refreshed, gradient
    zeroed), and full steps (fused train launch + Adam) timed end to end."""
    from qsdvr_b200 import fused
    from qsdvr_b200.optim import adam_step

    def timed(fn, reps):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    zero_ms = timed(lambda: (sg.zero_(), dg.zero_()), 5)
    # the share of parameters one step's gradient touches (non-zero after one train launch)
    sg.zero_(), dg.zero_()
    b0 = batches[0]
    order0 = fused.ray_order(b0["rays"], b0["origin"], b0["dir"], cfg["interval"])
    fused.render_train(b0["target"], b0["rays"], b0["origin"], b0["dir"], sdf_k, data_k, cfg["R"], cfg["interval"],
                       K_LOGISTIC, sg, dg, mode, transmittance, loss=loss, color=color, order=order0)
    touched_rows = float((dg.reshape(dg.shape[0], -1) != 0).any(1).float().mean())
    touched = float(((sg != 0).sum() + (dg != 0).sum()) / (sg.numel() + dg.numel()))
    params = [sdf.clone(), data.clone()]
    grads = [sg, dg]
    moments = [(torch.zeros_like(q), torch.zeros_like(q)) for q in params]
    moments16 = [(torch.zeros_like(q, dtype=torch.bfloat16), torch.zeros_like(q, dtype=torch.bfloat16))
                 for q in params]
    copies = [sdf_k, data_k] if sdf_k.dtype == torch.bfloat16 else [None, None]
    count = [0]

    def adam(state=moments, lazy=False, zero=True):
        count[0] += 1
        for j, (q, g, (m, v), c) in enumerate(zip(params, grads, state, copies)):
            adam_step(q, g, m, v, count[0], 1e-3, param_bf16=c, sdf_cells=(j == 0), skip_zero_grad=lazy,
                      zero_grad=zero)

    adam_ms = timed(adam, 5)
    adam16_ms = timed(lambda: adam(moments16), 5)
    # the lazy step on one real gradient (not zeroed in between, so each repetition sees it)
    fused.render_train(b0["target"], b0["rays"], b0["origin"], b0["dir"], sdf_k, data_k, cfg["R"], cfg["interval"],
                       K_LOGISTIC, sg, dg, mode, transmittance, loss=loss, color=color, order=order0)
    lazy_ms = timed(lambda: adam(lazy=True, zero=False), 5)
    sg.zero_(), dg.zero_()

    def full(state=moments):
        b = batches[count[0] % len(batches)]
        loss.zero_()
        order = fused.ray_order(b["rays"], b["origin"], b["dir"], cfg["interval"])
        fused.render_train(b["target"], b["rays"], b["origin"], b["dir"], sdf_k, data_k, cfg["R"], cfg["interval"],
                           K_LOGISTIC, sg, dg, mode, transmittance, loss=loss, color=color, order=order,
                           merge=args.merge)
        adam(state)

    full_ms = timed(full, max(3, args.steps // 2))
    full16_ms = timed(lambda: full(moments16), max(3, args.steps // 2))
    del params, moments, moments16
    return {"zero_grad_ms": round(zero_ms, 4), "adam_ms": round(adam_ms, 4),
            "adam_bf16_state_ms": round(adam16_ms, 4), "adam_lazy_ms": round(lazy_ms, 4),
            "touched_param_fraction": round(touched, 4), "touched_vertex_row_fraction": round(touched_rows, 4),
            "full_step_ms": round(full_ms, 4), "full_step_rays_per_s": round(cfg["rays"] / (full_ms / 1e3), 1),
            "full_step_bf16_state_ms": round(full16_ms, 4),
            "full_step": "fused forward/MSE/backward + fused Adam over both grids (fp32 masters; bf16 copies "
                         "refreshed for bf16 storage; gradients zeroed in the same pass)"}


# ----------------------------------------------------------------------------- proposal path

def proposal_comparison(steps: int, warmup_frac: float = 0.2, interval: float = 4.0 / 256, storage: str = "f32"):
    """Training at 256^3 from the same initial model on the same ray pool: the uniform march
    (4 / interval samples/ray, 65536 rays/step) and the proposal path (64 coarse MLP points + 32 fine
    samples/ray, network trained online every step; twice the rays per step, which costs
    about the render time of one plain step; the first ``warmup_frac`` of its steps use the
    uniform march while the network learns).  rays/s is device time of the forward + backward part of the
    steps (for the proposal: coarse MLP, sampler, online network update and the fused train
    launch); PSNR is on 65536 held-out rays rendered by the uniform march."""
    from qsdvr_b200 import train

    a = train.parser().parse_args([])
    a.steps, a.log_every, a.interval, a.storage = steps, 10 ** 9, interval, storage
    data = train.build(a.reso, a.views, a.size, 1111.1 * a.size / 800, 4.03, a.interval, a.k, a.seed,
                       torch.device("cuda", torch.cuda.current_device()))
    plain = train.run(a, data, quiet=True)
    a.proposal, a.rays, a.proposal_mix, a.proposal_warmup = True, 2 * a.rays, 0.05, int(round(steps * warmup_frac))
    prop = train.run(a, data, quiet=True)
    del data
    torch.cuda.empty_cache()
    return {"method": "64 coarse MLP points + 32 fine samples per ray (tcgen05 MLP, trained online)",
            "workload": f"R={a.reso}^3 {'fp32' if storage == 'f32' else 'bf16 storage (fp32 masters)'} fixed "
                        f"mode, {steps} training steps per method from the same sphere "
                        f"init, k={a.k}, Adam lr {a.lr}; plain {plain['rays_per_step']} rays/step, proposal "
                        f"{prop['rays_per_step']} rays/step with {a.proposal_warmup} uniform warm-up steps",
            "train_rays_per_s": prop["render_rays_per_s"], "plain_train_rays_per_s": plain["render_rays_per_s"],
            "speedup": round(prop["render_rays_per_s"] / plain["render_rays_per_s"], 3),
            "steady_train_rays_per_s": prop["steady_render_rays_per_s"],
            "steady_speedup": round(prop["steady_render_rays_per_s"] / plain["render_rays_per_s"], 3),
            "render_ms_per_step": round(prop["render_ms"] / steps, 4),
            "plain_render_ms_per_step": round(plain["render_ms"] / steps, 4),
            "optimizer_ms_per_step": round(prop["optimizer_ms"] / steps, 4),
            "psnr_plain": plain["heldout_psnr_end"], "psnr_proposal": prop["heldout_psnr_end"],
            "delta_psnr": round(plain["heldout_psnr_end"] - prop["heldout_psnr_end"], 3),
            "psnr_proposal_render": prop["heldout_psnr_end_proposal_render"],
            "delta_psnr_method": round(plain["heldout_psnr_end"] - prop["heldout_psnr_end_proposal_render"], 3),
            "psnr_reference": "held-out rays vs ground truth: delta_psnr with both models rendered by the 256-sample "
                     "uniform march, delta_psnr_method with each model rendered by its own method"}


# algorithmic FLOPs of the 32 -> 64 -> 64 -> 1 network per point (padding of the tensor-core
# tiles not counted): layer 1 and 2 GEMMs, b2, the head; training adds dH1, dW2, dW1 and the
# head / bias gradients
MLP_FLOPS_PER_POINT = 2 * 32 * 64 + 2 * 64 * 64 + 3 * 64
MLP_TRAIN_FLOPS_PER_POINT = MLP_FLOPS_PER_POINT + 2 * 64 * 64 + 2 * 64 * 64 + 2 * 32 * 64 + 4 * 64


def run_mlp_kernels(args, cfg, device):
    """Coarse MLP inference over a 65536-ray batch (4.2 M points) timed over K launches, with
    the tensor roofline; the other proposal kernels and both render modes timed beside it."""
    from qsdvr_b200 import fused, proposal, scenes, train

    R, interval, k = cfg["R"], cfg["interval"], 5.0
    rays, origin, direction, target = train.build(R, cfg["views"], cfg["size"], cfg["focal"], cfg["radius"],
                                                  interval, k, 0, device)
    sdf = fused.pad_grid7(scenes.procedural_grid(R, seed=0, device=device).reshape(-1, 7))
    data = scenes.appearance(R, seed=0, device=device, procedural=True)
    gen = torch.Generator(device=device).manual_seed(0)
    idx = torch.randint(0, rays.shape[0], (cfg["rays"],), generator=gen, device=device)
    r, o, d, tg = (t[idx].contiguous() for t in (rays, origin, direction, target))
    net = proposal.ProposalNet(device)
    for _ in range(cfg["online_steps"]):
        net.online_step(r[:4096], o[:4096], d[:4096], sdf, data, R, interval, k)
    stream = torch.cuda.current_stream(device)

    def timed(fn):
        def step(i, ev):
            if ev is not None:
                ev[0].record(stream)
            fn()
            if ev is not None:
                ev[1].record(stream)
        return time_device(step, args.steps, args.warmup, stream)[0] / args.steps

    with ClockSampler(device.index) as clk:
        time.sleep(0.3)
        infer_ms = timed(lambda: net.coarse_density(r, o, d, interval))
    coarse = net.coarse_density(r, o, d, interval)
    tl = proposal.sample_fine(r, interval, coarse)
    pts = torch.rand((cfg["rays"], 4), generator=gen, device=device)
    sg, dg = torch.zeros_like(sdf), torch.zeros_like(data)
    side = {
        "sample_ms": timed(lambda: proposal.sample_fine(r, interval, coarse)),
        "mlp_train_65536_points_ms": timed(lambda: net.gradients(pts)),
        "online_step_4096_rays_ms": timed(lambda: net.online_step(r[:4096], o[:4096], d[:4096], sdf, data, R,
                                                                  interval, k)),
        "list_train_ms": timed(lambda: fused.render_train(tg, r, o, d, sdf, data, R, interval, k, sg, dg, "fixed",
                                                          tlist=tl)),
        # rays taken by the Morton order of their median fine sample (qsdvr_ray_order_list, as
        # in training), the order computed inside the timed launch sequence
        "list_train_ordered_ms": timed(lambda: fused.render_train(
            tg, r, o, d, sdf, data, R, interval, k, sg, dg, "fixed", tlist=tl,
            order=fused.ray_order(r, o, d, interval, tlist=tl))),
        "uniform_train_ordered_ms": timed(lambda: fused.render_train(
            tg, r, o, d, sdf, data, R, interval, k, sg, dg, "fixed", order=fused.ray_order(r, o, d, interval))),
        "uniform_train_ms": timed(lambda: fused.render_train(tg, r, o, d, sdf, data, R, interval, k, sg, dg,
                                                             "fixed")),
        "list_forward_ms": timed(lambda: fused.render_forward(r, o, d, sdf, data, R, interval, k, "fixed",
                                                              tlist=tl)),
        "uniform_forward_ms": timed(lambda: fused.render_forward(r, o, d, sdf, data, R, interval, k, "fixed")),
    }
    side["mlp_train_tflops"] = round(cfg["rays"] * MLP_TRAIN_FLOPS_PER_POINT / (side["mlp_train_65536_points_ms"]
                                                                               * 1e-3) / 1e12, 1)
    side = {kk: (round(v, 4) if isinstance(v, float) else v) for kk, v in side.items()}
    hit = int((r[:, 0] >= 2).sum())
    points = cfg["rays"] * 64
    tflops = points * MLP_FLOPS_PER_POINT / (infer_ms * 1e-3) / 1e12
    peak = measured_peak_tensor()
    return {
        "metric": "proposal MLP coarse-density inference points/s (64 points per ray)",
        "value": round(points / (infer_ms * 1e-3), 1), "unit": "points/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(infer_ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16 (f32 accumulation)", "data": "synthetic (seeded procedural scene)",
        "config": {"workload": f"mlp256: 32-d encoding -> 64 -> 64 -> 1 on {cfg['rays']} rays of the {R}^3 scene "
                               f"({hit} with samples), network trained online for {cfg['online_steps']} steps",
                   "global_batch": points, "l2": "weights in shared memory; inputs 1.6 MB, no flush",
                   "parallelism": "replicas x1"},
        "gpu_launches": args.steps,
        "roofline": {"bound": "tensor", "achieved": round(tflops, 1), "peak": peak[0], "unit": "TFLOP/s",
                     "frac": round(tflops / peak[0], 4), "traffic": None, "kernel": "mlp_infer_kernel",
                     "flops_per_point": MLP_FLOPS_PER_POINT, "peak_kind": peak[1]},
        "kernels": side, "clocks": clk.summary(),
    }


def run_train512(args, cfg, device):
    """The default line's proposal comparison with the uniform march at 512 samples/ray (the
    learned proposal form's reference march) on the 256^3 scene."""
    cmp = proposal_comparison(PROPOSAL_STEPS, args.proposal_warmup, cfg["interval"])
    return {
        "metric": "train rays/s fwd+bwd @256^3: proposal (64 coarse + 32 fine) vs 512-sample uniform march",
        "value": cmp["train_rays_per_s"], "unit": "rays/s", "n_gpus": 1, "steps": PROPOSAL_STEPS,
        "warmup": int(round(PROPOSAL_STEPS * args.proposal_warmup)), "ms_per_step": cmp["render_ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded procedural scene; model trained from a sphere init)",
        "config": {"workload": "train512: " + cmp["workload"] + ", interval 4/512",
                   "global_batch": 2 * cfg["rays"], "parallelism": "replicas x1"},
        "gpu_launches": None, "proposal": cmp,
    }


def measured_peak_tensor():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured (burst)"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback"


def run_proposal_frames(args, cfg, device):
    """Learned proposal form: train a BF16 SH3 model (uniform march, proposal network trained
    online beside it), then render held-out full frames with the 512-sample uniform march and
    with 64 coarse MLP points + 32 fine samples per ray; rays/s (all pixels) and PSNR of each
    against the ground-truth frames."""
    from qsdvr_b200 import fused, scenes, train
    from qsdvr_b200.camera import Camera

    R, interval = cfg["R"], cfg["interval"]
    a = train.parser().parse_args([])
    a.reso, a.interval, a.sh, a.storage, a.views = R, interval, cfg["sh"], cfg["storage"], cfg["views"]
    a.steps, a.rays, a.log_every, a.online_proposal = cfg["train_steps"], cfg["rays"], 10 ** 9, True
    size = cfg["size"]
    data = train.build(R, a.views, size, cfg["focal"], cfg["radius"], interval, a.k, a.seed, device, a.sh)
    summary, model, net = train.run(a, data, quiet=True, return_state=True)
    del data
    torch.cuda.empty_cache()
    # held-out views (a different camera seed) and their ground truth from the uniform march
    gt_sdf = fused.pad_grid7(scenes.procedural_grid(R, seed=a.seed, device=device).reshape(-1, 7))
    gt_data = scenes.appearance(R, seed=a.seed, device=device, procedural=True, sh_degree=a.sh)
    frames = []
    for cam in scenes.hemisphere_cameras(cfg["heldout"], cfg["radius"], size, size, cfg["focal"], 2.0, 6.0,
                                         seed=a.seed + 99):
        c = Camera(cam, interval, R, device=device)
        c.GenerateRayPoints(torch.ones(size * size, dtype=torch.bool), order=args.ray_order)
        gt = fused.render_forward(c.rayList, c.originList, c.dirList, gt_sdf, gt_data, R, interval, a.k, "fixed")
        frames.append((c.rayList, c.originList, c.dirList, gt))
    del gt_sdf, gt_data
    torch.cuda.empty_cache()
    sg, dg = model.grids()
    sg, dg = sg.detach(), dg.detach()
    stream = torch.cuda.current_stream(device)

    def uniform(f):
        return fused.render_forward(f[0], f[1], f[2], sg, dg, R, interval, a.k, "fixed", model.transmittance)

    def proposal(f):
        return net.render(f[0], f[1], f[2], sg, dg, R, interval, a.k, "fixed", model.transmittance)

    out = {}
    for name, fn in (("uniform", uniform), ("proposal", proposal)):
        mse = sum(float(((fn(f) - f[3]) ** 2).mean()) for f in frames) / len(frames)

        def step(i, ev, fn=fn):
            if ev is not None:
                ev[0].record(stream)
            fn(frames[i % len(frames)])
            if ev is not None:
                ev[1].record(stream)

        with ClockSampler(device.index) as clk:
            time.sleep(0.3)
            total_ms, kern_ms = time_device(step, args.steps, args.warmup, stream, clk)
        out[name] = dict(ms_per_frame=total_ms / args.steps, psnr=-10.0 * np.log10(max(mse, 1e-12)),
                         clocks=clk.summary())
    # the brick-staged forward (TMA bricks of the appearance grid, one thread per ray) against
    # the fused forward, both on the same frames listed tile by tile (8 x 8 pixels)
    tiled = []
    for cam in scenes.hemisphere_cameras(cfg["heldout"], cfg["radius"], size, size, cfg["focal"], 2.0, 6.0,
                                         seed=a.seed + 99):
        c = Camera(cam, interval, R, device=device)
        c.GenerateRayPoints(torch.ones(size * size, dtype=torch.bool), order="tiles")
        tiled.append((c.rayList, c.originList, c.dirList))
    bricks = {}
    diff = 0.0
    for f in tiled:
        diff = max(diff, float((fused.render_forward_bricks(f[0], f[1], f[2], sg, dg, R, interval, a.k)
                                - uniform(f)).abs().max()))
    for name, fn in (("fused_forward_tiles", uniform),
                     ("brick_forward_tiles", lambda f: fused.render_forward_bricks(f[0], f[1], f[2], sg, dg, R,
                                                                                   interval, a.k))):
        def bstep(i, ev, fn=fn):
            if ev is not None:
                ev[0].record(stream)
            fn(tiled[i % len(tiled)])
            if ev is not None:
                ev[1].record(stream)

        bricks[name + "_ms"] = round(time_device(bstep, args.steps, args.warmup, stream)[0] / args.steps, 4)
    bricks["max_abs_colour_difference"] = diff
    pixels = size * size
    value = pixels / (out["proposal"]["ms_per_frame"] / 1e3)
    plain = pixels / (out["uniform"]["ms_per_frame"] / 1e3)
    return {
        "metric": "full-frame render rays/s, proposal (64 coarse + 32 fine) vs 512-sample uniform march",
        "value": round(value, 1), "unit": "rays/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(out["proposal"]["ms_per_frame"], 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16 storage, f32 math; MLP bf16 with f32 accumulation",
        "data": "synthetic (seeded procedural scene; model trained from a sphere init)",
        "config": {"workload": f"{args.workload}: R={R}^3 BF16 SH3 model after {a.steps} training steps "
                               f"({a.rays} rays/step, uniform 512 march, proposal network trained online), "
                               f"{cfg['heldout']} held-out {size}^2 frames, k={a.k}",
                   "global_batch": pixels, "step": "one full frame (all pixels, hit or not)",
                   "ray_order": args.ray_order,
                   "l2": "grids 8.2 GB, larger than L2; no flush", "parallelism": "replicas x1"},
        "plain_value": round(plain, 1), "speedup": round(value / plain, 3),
        "psnr_uniform512": round(out["uniform"]["psnr"], 3), "psnr_proposal": round(out["proposal"]["psnr"], 3),
        "delta_psnr": round(out["uniform"]["psnr"] - out["proposal"]["psnr"], 3),
        "train_summary": {k: summary[k] for k in ("heldout_psnr_end", "ms_per_step", "peak_memory_gb")},
        "gpu_launches": 3 * args.steps, "clocks": out["proposal"]["clocks"],
        "brick_staging": bricks,
    }


# ----------------------------------------------------------------------------- CPU path

def _cpu_step(grid7, data, batch_cpu, R, interval):
    """One fwd+bwd of the reference's torch render path on the host (its per-ray loop)."""
    from oracle.render_torch_cpu import render_torch_cpu
    from qsdvr_b200.qsdvr import CameraArgs  # noqa: F401  (same package, no GPU use)
    import oracle.oracle as O

    pts = O.generate_ray_points(batch_cpu["rays"], batch_cpu["origin"], batch_cpu["dir"], interval, R)
    inp = {k: torch.from_numpy(v) for k, v in pts.items()}
    inp["rayList"] = torch.from_numpy(batch_cpu["rays_packed"].astype(np.int64))
    g = grid7.detach().requires_grad_()
    d = data.detach().requires_grad_()
    img = render_torch_cpu(g, d, inp, R, K_LOGISTIC)
    loss = ((img - batch_cpu["target"]) ** 2).mean()
    loss.backward()
    return float(loss)


def _oracle_step(grid7, data, batch_cpu, R, interval):
    """The same fwd+bwd by the float64 vectorised oracle (oracle/oracle.py, torch autograd)."""
    import oracle.oracle as O

    pts = O.generate_ray_points(batch_cpu["rays"], batch_cpu["origin"], batch_cpu["dir"], interval, R)
    inp = {k: torch.from_numpy(v) for k, v in pts.items()}
    inp["rayList"] = torch.from_numpy(batch_cpu["rays_packed"].astype(np.int64))
    g = grid7.detach().double().requires_grad_()
    d = data.detach().double().requires_grad_()
    img = O.render(g, d, inp, K_LOGISTIC, compat=True)
    loss = ((img - batch_cpu["target"].double()) ** 2).mean()
    loss.backward()
    return float(loss)


def _cpu_batch(batch, n):
    """First n rays of a batch, repacked with fresh sample offsets (host arrays)."""
    rays = batch["rays"][:n].cpu().numpy().view(np.uint32).copy()
    c = rays[:, 0].astype(np.int64)
    rc = np.maximum(c - 1, 0)
    rays[:, 1] = np.cumsum(c) - c
    rays[:, 2] = rc
    rays[:, 3] = np.cumsum(rc) - rc
    return dict(rays=rays, rays_packed=rays, origin=batch["origin"][:n].cpu().numpy(),
                dir=batch["dir"][:n].cpu().numpy(), target=batch["target"][:n].cpu())


def cpu_baseline(scene, batch, cfg, n_rays, steps=1):
    """The reference's CPU path on a bounded sample: n_rays of one batch, fwd+bwd."""
    sdf, data = scene["model"]
    grid7 = sdf[:, :7].contiguous().cpu()
    data_cpu = data.cpu()
    b = _cpu_batch(batch, n_rays)
    threads = torch.get_num_threads()
    _cpu_step(grid7, data_cpu, b, cfg["R"], cfg["interval"])  # warm-up
    t0 = time.perf_counter()
    for _ in range(steps):
        _cpu_step(grid7, data_cpu, b, cfg["R"], cfg["interval"])
    dt = (time.perf_counter() - t0) / steps
    return {"value": round(n_rays / dt, 2), "unit": "rays/s", "cores": threads, "kind": "port",
            "sample": f"{n_rays} rays of one {cfg['rays']}-ray batch ({int(np.maximum(b['rays'][:, 0].astype(np.int64) - 1, 0).sum())} "
                      f"render samples), fwd+bwd of the reference's torch render path (models/render_torch.py "
                      f"per-ray loop) on the host, {steps} timed step(s) after 1 warm-up; os.cpu_count()="
                      f"{os.cpu_count()}"}


def reference_batch_cpu(cfg, n_rays, seed=0):
    """A bounded sample of the workload built on the host alone, with the oracle: the model
    grids of the GPU arm (same seeds), ``n_rays`` pixels drawn at random over the same seeded
    views and marched by the oracle's RayCut (oracle/raygen.c), and their targets rendered by
    the oracle (float32, fixed mode) from the ground-truth scene.  config1 takes every pixel of
    its one view and a seeded U(0,1) target image.  Nothing here loads the product library."""
    import oracle.oracle as O
    from qsdvr_b200 import scenes

    R = cfg["R"]
    if cfg.get("scene") == "sphere":
        a = scenes.look_at(CONFIG1_CAMERA, cfg["size"], cfg["size"], cfg["focal"], 2.0, 6.0)
        cam = O.Camera(a.width, a.height, tuple(a.rotation), tuple(a.translation), a.fx, a.fy, a.cx, a.cy, a.near,
                       a.far)
        rays, origin, direction, _, _ = O.ray_cut(cam, np.ones(a.width * a.height, np.uint8), cfg["interval"])
        grid7 = scenes.sphere_grid(R, 0.5, 0.01, seed=seed).reshape(-1, 7).contiguous()
        data = scenes.appearance(R, seed=seed)
        target = torch.rand((rays.shape[0], 3), generator=torch.Generator().manual_seed(0))
        return grid7, data, dict(rays=rays, rays_packed=rays, origin=origin, dir=direction, target=target)
    cams = scenes.hemisphere_cameras(cfg["views"], cfg["radius"], cfg["size"], cfg["size"], cfg["focal"], 2.0, 6.0,
                                     seed=seed)
    rng = np.random.default_rng(1000 + seed)
    views = rng.integers(0, len(cams), n_rays)
    pixels = rng.integers(0, cfg["size"] * cfg["size"], n_rays)
    rays = np.zeros((n_rays, 4), np.uint32)
    origin = np.zeros((n_rays, 3), np.float32)
    direction = np.zeros((n_rays, 3), np.float32)
    for i, (v, px) in enumerate(zip(views, pixels)):
        a = cams[v]
        cam = O.Camera(a.width, a.height, tuple(a.rotation), tuple(a.translation), a.fx, a.fy, a.cx, a.cy, a.near,
                       a.far)
        r, o, d = O.ray_cut_pixels(cam, np.array([px], np.uint32), cfg["interval"])
        rays[i], origin[i], direction[i] = r[0], o[0], d[0]
    c = rays[:, 0].astype(np.int64)
    rc = np.maximum(c - 1, 0)
    rays[:, 1] = np.cumsum(c) - c
    rays[:, 2] = rc
    rays[:, 3] = np.cumsum(rc) - rc
    pts = O.generate_ray_points(rays, origin, direction, cfg["interval"], R)
    inp = {k: torch.from_numpy(v) for k, v in pts.items()}
    inp["rayList"] = torch.from_numpy(rays.astype(np.int64))
    gt7 = scenes.procedural_grid(R, seed=seed).reshape(-1, 7)
    gt_data = scenes.appearance(R, seed=seed, procedural=True)
    with torch.no_grad():
        target = O.render(gt7, gt_data, inp, K_LOGISTIC, compat=False).float()
    del gt7, gt_data
    grid7 = scenes.sphere_grid(R, 0.5, 0.01, seed=seed).reshape(-1, 7).contiguous()
    data = scenes.appearance(R, seed=seed + 1)
    return grid7, data, dict(rays=rays, rays_packed=rays, origin=origin, dir=direction, target=target)


def run_reference(args, cfg):
    """The reference's CPU implementation timed on the host cores (rank 0 only); its batch is
    built on the host by the oracle (reference_batch_cpu)."""
    if cfg.get("sh", 2) != 2:
        print(json.dumps({"impl": "reference", "unavailable": "the reference renders SH degree 2 only"}))
        return
    torch.set_num_threads(os.cpu_count() or 1)
    n = cfg["rays"] if cfg.get("scene") == "sphere" else args.cpu_rays
    grid7, data_cpu, b = reference_batch_cpu(cfg, n)
    n = b["rays"].shape[0]
    for _ in range(args.warmup):
        _cpu_step(grid7, data_cpu, b, cfg["R"], cfg["interval"])
    t0 = time.perf_counter()
    for _ in range(args.steps):
        _cpu_step(grid7, data_cpu, b, cfg["R"], cfg["interval"])
    dt = time.perf_counter() - t0
    value = n * args.steps / dt
    # the float64 oracle on the same sample, one step after a warm-up: reported beside the
    # baseline, not as it
    _oracle_step(grid7, data_cpu, b, cfg["R"], cfg["interval"])
    t1 = time.perf_counter()
    _oracle_step(grid7, data_cpu, b, cfg["R"], cfg["interval"])
    oracle_rays_per_s = n / (time.perf_counter() - t1)
    samples = int(np.maximum(b["rays"][:, 0].astype(np.int64) - 1, 0).sum())
    full = cfg.get("scene") == "sphere"
    sample = (f"all {n} rays of the view ({samples} render samples)" if full else
              f"{n} rays per step drawn at random over the {cfg['views']} views ({samples} render samples) of the "
              f"{cfg['rays']}-ray batch's ray pool")
    # n_gpus mirrors the launch (--gpus N); the timed work runs on rank 0's host cores
    line = {"metric": METRIC, "impl": "reference", "value": round(value, 2), "unit": "rays/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (the GPU arm's seeded scene; rays and targets made on the host by the oracle)",
            "config": {"workload": f"{args.workload}: " + ("full case" if full else "bounded sample") + f", {sample}",
                       "global_batch": n},
            "cpu_baseline": {"value": round(value, 2), "unit": "rays/s", "cores": torch.get_num_threads(),
                             "kind": "port",
                             "sample": f"{sample}; reference torch render path (models/render_torch.py, per-ray "
                                       f"loop) fwd+bwd on the host; os.cpu_count()={os.cpu_count()}"},
            "e2e": {"value": round(value, 2), "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "oracle_timing": {"value": round(oracle_rays_per_s, 2), "unit": "rays/s",
                              "label": "oracle, not the baseline: the float64 vectorised restatement "
                                       "(oracle/oracle.py, compat mode, torch autograd) fwd+bwd on the same sample"}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="plain256", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-rays", type=int, default=48)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--merge", action="store_true",
                    help="same-cell merged appearance scatter (samples of a chunk in one cell send one RED per row)")
    ap.add_argument("--no-proposal", action="store_true", help="skip the proposal-path comparison")
    ap.add_argument("--proposal-warmup", type=float, default=0.2,
                    help="fraction of the proposal run's steps trained with the uniform march first")
    ap.add_argument("--views", type=int, default=None, help="override the number of camera views (ray pool size)")
    ap.add_argument("--ray-order", default="pixels", choices=["pixels", "tiles"],
                    help="order of a full frame's rays (proposal384): row-major pixels or 8x8 tiles")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    cfg = dict(WORKLOADS[args.workload])
    if args.views:
        cfg["views"] = args.views
    ws, rank, local = dist_env()
    if args.impl == "reference":
        if rank == 0:
            run_reference(args, cfg)
        return
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if ws > 1:
        import datetime

        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=device)
    try:
        if args.workload in ("proposal384", "proposal128", "mlp256", "mlp128", "train512"):
            if ws > 1:
                raise SystemExit(f"{args.workload} is a single-GPU workload")
            fn = {"proposal384": run_proposal_frames, "proposal128": run_proposal_frames, "mlp256": run_mlp_kernels,
                  "mlp128": run_mlp_kernels, "train512": run_train512}[args.workload]
            print(json.dumps(fn(args, cfg, device)))
            return
        out = run_ours(args, cfg, device, ws, rank)
        if rank == 0:
            print(json.dumps(out))
    finally:
        if ws > 1:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
