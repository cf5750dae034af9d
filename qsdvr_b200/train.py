"""Training loop on a seeded synthetic scene with the fused kernels (test.py:16-37's loop:
random ray batches, forward + MSE + backward, Adam), reporting loss, PSNR on held-out
rays, step time and peak device memory.

    python -m qsdvr_b200.train --reso 256 --steps 1000 --rays 65536 --lr 1e-2

Targets come from a seeded procedural ground-truth scene rendered once for every pixel of
every view; the model starts from a sphere SDF and constant appearance (models/render.py:
215-223).  Per-sample values are recomputed in the backward, so memory beyond the grids,
their gradients and Adam state is O(rays).
"""
from __future__ import annotations

import argparse
import json
import math
import time

import torch

from . import fused, scenes
from .camera import Camera
from .optim import FusedGridAdam


def build(reso, views, size, focal, radius, interval, k, seed, device):
    gt_sdf = fused.pad_grid7(scenes.procedural_grid(reso, seed=seed, device=device).reshape(-1, 7))
    gt_data = scenes.appearance(reso, seed=seed, device=device, procedural=True)
    cams = scenes.hemisphere_cameras(views, radius, size, size, focal, 2.0, 6.0, seed=seed)
    rays, origin, direction, target = [], [], [], []
    mask = torch.ones(size * size, dtype=torch.bool)
    for a in cams:
        c = Camera(a, interval, reso, device=device)
        c.GenerateRayPoints(mask)
        rays.append(c.rayList)
        origin.append(c.originList)
        direction.append(c.dirList)
        target.append(fused.render_forward(c.rayList, c.originList, c.dirList, gt_sdf, gt_data, reso, interval, k,
                                           "fixed"))
    del gt_sdf, gt_data
    return torch.cat(rays), torch.cat(origin), torch.cat(direction), torch.cat(target)


def psnr(mse: float) -> float:
    return -10.0 * math.log10(max(mse, 1e-12))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reso", type=int, default=256)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--rays", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-2)
    ap.add_argument("--views", type=int, default=100)
    ap.add_argument("--size", type=int, default=800)
    ap.add_argument("--interval", type=float, default=4.0 / 256)
    ap.add_argument("--k", type=float, default=5.0)
    ap.add_argument("--storage", default="f32", choices=["f32", "bf16"])
    ap.add_argument("--mode", default="fixed", choices=["fixed", "compat"])
    ap.add_argument("--log-every", type=int, default=100)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    dev = torch.device("cuda", torch.cuda.current_device())
    R = a.reso
    rays, origin, direction, target = build(R, a.views, a.size, 1111.1 * a.size / 800, 4.03, a.interval, a.k, a.seed,
                                            dev)
    total = rays.shape[0]
    gen = torch.Generator(device=dev).manual_seed(a.seed + 1)
    held = torch.randint(0, total, (a.rays,), generator=gen, device=dev)
    torch.cuda.reset_peak_memory_stats(dev)
    base_mem = torch.cuda.memory_allocated(dev)
    model = fused.DenseRenderGrid(R, a.k, a.interval, mode=a.mode, storage=a.storage, device=dev)
    copies = dict(zip((model.sdfGrid, model.renderData), model._copies)) if a.storage == "bf16" else None
    opt = FusedGridAdam(model.parameters(), lr=a.lr, bf16_copies=copies)
    model.sdfGrid.grad = torch.zeros_like(model.sdfGrid)
    model.renderData.grad = torch.zeros_like(model.renderData)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    log = []

    def evaluate():
        sg, dg = model.grids()
        col = fused.render_forward(rays[held], origin[held], direction[held], sg.detach(), dg.detach(), R, a.interval,
                                   a.k, a.mode, model.transmittance)
        return float(((col - target[held]) ** 2).mean())

    start_mse = evaluate()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for step in range(1, a.steps + 1):
        idx = torch.randint(0, total, (a.rays,), generator=gen, device=dev)
        sg, dg = model.grids()
        loss.zero_()
        fused.render_train(target[idx], rays[idx], origin[idx], direction[idx], sg.detach(), dg.detach(), R,
                           a.interval, a.k, model.sdfGrid.grad, model.renderData.grad, a.mode, model.transmittance,
                           loss=loss)
        opt.step()  # Adam on the fp32 masters; zeroes the gradients, refreshes bf16 copies
        if step % a.log_every == 0 or step == a.steps:
            torch.cuda.synchronize()
            mse = float(loss) / (3 * a.rays)
            log.append({"step": step, "train_mse": mse, "elapsed_s": round(time.perf_counter() - t0, 3)})
            print(json.dumps(log[-1]), flush=True)
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    end_mse = evaluate()
    out = {"reso": R, "steps": a.steps, "rays_per_step": a.rays, "lr": a.lr, "storage": a.storage, "mode": a.mode,
           "ms_per_step": round(1e3 * elapsed / a.steps, 3), "train_rays_per_s": round(a.steps * a.rays / elapsed),
           "heldout_psnr_start": round(psnr(start_mse), 3), "heldout_psnr_end": round(psnr(end_mse), 3),
           "peak_memory_gb": round(torch.cuda.max_memory_allocated(dev) / 1e9, 3),
           "model_and_state_gb": round((torch.cuda.max_memory_allocated(dev) - base_mem) / 1e9, 3),
           "ray_pool_gb": round(base_mem / 1e9, 3)}
    print(json.dumps(out), flush=True)
    return out


if __name__ == "__main__":
    main()
