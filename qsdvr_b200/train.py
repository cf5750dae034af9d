"""Training loop on a seeded synthetic scene with the fused kernels (test.py:16-37's loop:
random ray batches, forward + MSE + backward, Adam), reporting loss, PSNR on held-out
rays, step time and peak device memory.

    python -m qsdvr_b200.train --reso 256 --steps 1000 --rays 65536 --lr 1e-2 [--proposal]

Targets come from a seeded procedural ground-truth scene rendered once for every pixel of
every view; the model starts from a sphere SDF and constant appearance (models/render.py:
215-223).  Per-sample values are recomputed in the backward, so memory beyond the grids,
their gradients and Adam state is O(rays).

``--proposal`` trains the grid at the proposal network's 32 fine samples per ray (64 coarse
MLP evaluations place them) instead of the uniform march (after ``--proposal-warmup`` steps
with it).  The network is trained online every step on the per-sample alphas of a
uniform-march forward over part of the batch.
Held-out PSNR is always measured with the uniform march.

``--model separable`` trains the reference's own parametrisation instead of a dense quadric
grid: the three per-axis layers and the offset of models/render.py:172-207 (Adam, as
test.py:20) with the appearance grid (fused Adam), through the fused kernels that assemble
cells from the layers' tables.

``--save PATH`` writes a checkpoint (checkpoint.py) at the end and every ``--save-every``
steps; ``--resume PATH`` continues a run from one, with the same ray batches as the run that
was not interrupted.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import torch

from . import checkpoint, fused, scenes
from .camera import Camera
from .optim import FusedGridAdam


def build(reso, views, size, focal, radius, interval, k, seed, device, sh_degree=2):
    gt_sdf = fused.pad_grid7(scenes.procedural_grid(reso, seed=seed, device=device).reshape(-1, 7))
    gt_data = scenes.appearance(reso, seed=seed, device=device, procedural=True, sh_degree=sh_degree)
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


def parser():
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
    ap.add_argument("--sh", type=int, default=2, choices=[2, 3])
    ap.add_argument("--proposal", action="store_true", help="train at the proposal network's fine samples")
    ap.add_argument("--online-proposal", action="store_true",
                    help="train the grid with the uniform march and the proposal network online beside it")
    ap.add_argument("--proposal-rays", type=int, default=4096, help="rays of the per-step uniform pass")
    ap.add_argument("--proposal-points", type=int, default=65536, help="MLP training points per step")
    ap.add_argument("--proposal-lr", type=float, default=5e-3)
    ap.add_argument("--proposal-mix", type=float, default=0.25, help="uniform share of the fine-sample pdf")
    ap.add_argument("--proposal-warmup", type=int, default=0,
                    help="steps trained with the uniform march (network trained online) before the proposal")
    ap.add_argument("--log-every", type=int, default=100)
    ap.add_argument("--save", default=None, help="checkpoint path written at the end (and every --save-every)")
    ap.add_argument("--save-every", type=int, default=0)
    ap.add_argument("--resume", default=None, help="checkpoint to continue from (steps counts the total)")
    ap.add_argument("--grad-storage", default="f32", choices=["f32", "bf16"],
                    help="accumulate the appearance gradient in bf16 (half its traffic; SDF gradient fp32)")
    ap.add_argument("--no-ray-order", dest="ray_order", action="store_false",
                    help="take each batch's rays in batch order instead of the Morton order of their midpoints")
    ap.add_argument("--model", default="dense", choices=["dense", "separable"],
                    help="dense quadric grid, or the reference's separable layers (RenderGrid)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--adam-state", default="f32", choices=["f32", "bf16"],
                    help="Adam moments in bf16 (stochastic rounding; 24 instead of 32 B per parameter and step)")
    ap.add_argument("--lazy-adam", action="store_true",
                    help="leave parameters whose gradient is exactly 0 untouched (their moments do not decay)")
    return ap


def run(a, data=None, quiet=False, return_state=False):
    """Train per ``a`` (parser() namespace).  ``data``: (rays, origin, dir, target) to reuse
    a built scene.  Returns the summary dict; its "render_ms" is the device time of the
    render part of the steps (forward + backward, and with a proposal network the coarse MLP,
    the sampler and the online network update), "optimizer_ms" that of the grid Adam steps.
    ``return_state``: also return the trained model and proposal network (or None)."""
    from .proposal import ProposalNet

    dev = torch.device("cuda", torch.cuda.current_device())
    R = a.reso
    if data is None:
        data = build(R, a.views, a.size, 1111.1 * a.size / 800, 4.03, a.interval, a.k, a.seed, dev, a.sh)
    if getattr(a, "model", "dense") == "separable":
        return run_separable(a, data, quiet, return_state)
    rays, origin, direction, target = data
    total = rays.shape[0]
    gen = torch.Generator(device=dev).manual_seed(a.seed + 1)
    held = torch.randint(0, total, (a.rays,), generator=gen, device=dev)
    torch.cuda.reset_peak_memory_stats(dev)
    base_mem = torch.cuda.memory_allocated(dev)
    model = fused.DenseRenderGrid(R, a.k, a.interval, mode=a.mode, storage=a.storage, device=dev, sh_degree=a.sh)
    copies = dict(zip((model.sdfGrid, model.renderData), model._copies)) if a.storage == "bf16" else None
    data_grad = None
    if getattr(a, "grad_storage", "f32") == "bf16":
        data_grad = torch.zeros(model.renderData.shape, dtype=torch.bfloat16, device=dev)
    opt = FusedGridAdam(model.parameters(), lr=a.lr, bf16_copies=copies,
                        grads={model.renderData: data_grad} if data_grad is not None else None,
                        sdf_cells=(model.sdfGrid,), skip_zero_grad=getattr(a, "lazy_adam", False),
                        state_dtype=torch.bfloat16 if getattr(a, "adam_state", "f32") == "bf16" else torch.float32)
    model.sdfGrid.grad = torch.zeros_like(model.sdfGrid)
    if data_grad is None:
        model.renderData.grad = data_grad = torch.zeros_like(model.renderData)
    net = ProposalNet(dev, seed=a.seed, lr=a.proposal_lr) if (a.proposal or a.online_proposal) else None
    first = 1
    if getattr(a, "resume", None):
        first = checkpoint.load(a.resume, model, opt, net, gen) + 1
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    log = []

    def evaluate():
        sg, dg = model.grids()
        args = (rays[held], origin[held], direction[held], sg.detach(), dg.detach(), R, a.interval, a.k, a.mode,
                model.transmittance)
        col = fused.render_forward(*args)
        out = {"uniform": float(((col - target[held]) ** 2).mean())}
        if net is not None:
            colp = net.render(*args)
            out["proposal"] = float(((colp - target[held]) ** 2).mean())
        return out

    start = evaluate()
    steps = range(first, a.steps + 1)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in steps]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for step in steps:
        idx = torch.randint(0, total, (a.rays,), generator=gen, device=dev)
        r, o, d, tg = rays[idx], origin[idx], direction[idx], target[idx]
        sg, dg = model.grids()
        sg, dg = sg.detach(), dg.detach()
        e0, e1, e2 = ev[step - first]
        e0.record()
        loss.zero_()
        tlist = None
        if net is not None:
            n = min(a.proposal_rays, a.rays)
            net.online_step(r[:n], o[:n], d[:n], sg, dg, R, a.interval, a.k, a.mode, model.transmittance,
                            points=a.proposal_points)
            if a.proposal and step > a.proposal_warmup:
                tlist = net.sample(r, o, d, a.interval, a.proposal_mix)
        order = fused.ray_order(r, o, d, a.interval, tlist=tlist) if a.ray_order else None
        fused.render_train(tg, r, o, d, sg, dg, R, a.interval, a.k, model.sdfGrid.grad, data_grad,
                           a.mode, model.transmittance, loss=loss, tlist=tlist, order=order)
        e1.record()
        opt.step()  # Adam on the fp32 masters; zeroes the gradients, refreshes bf16 copies
        e2.record()
        if not quiet and (step % a.log_every == 0 or step == a.steps):
            torch.cuda.synchronize()
            mse = float(loss) / (3 * a.rays)
            log.append({"step": step, "train_mse": mse, "elapsed_s": round(time.perf_counter() - t0, 3)})
            print(json.dumps(log[-1]), flush=True)
        if getattr(a, "save", None) and ((a.save_every and step % a.save_every == 0) or step == a.steps):
            checkpoint.save(a.save, model, opt, net, step, gen)
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    render_ms = sum(e0.elapsed_time(e1) for e0, e1, _ in ev)
    opt_ms = sum(e1.elapsed_time(e2) for _, e1, e2 in ev)
    warm = max(0, (a.proposal_warmup if a.proposal else 0) - (first - 1))
    steady = [e0.elapsed_time(e1) for e0, e1, _ in ev[warm:]]
    end = evaluate()
    ran = len(steps)  # steps run in this call (all of them unless resumed)
    out = {"reso": R, "steps": a.steps, "first_step": first, "rays_per_step": a.rays, "lr": a.lr, "storage": a.storage, "mode": a.mode,
           "sh_degree": a.sh, "k": a.k,
           "method": "proposal 64 coarse + 32 fine" if a.proposal else
                     "uniform march" + (" + online proposal network" if net else ""),
           "ms_per_step": round(1e3 * elapsed / max(ran, 1), 3),
           "train_rays_per_s": round(ran * a.rays / elapsed) if ran else None,
           "render_ms": round(render_ms, 3), "optimizer_ms": round(opt_ms, 3),
           "render_rays_per_s": round(ran * a.rays / (render_ms / 1e3)) if ran else None,
           "steady_render_rays_per_s": round(len(steady) * a.rays / (sum(steady) / 1e3)) if steady else None,
           "heldout_psnr_start": round(psnr(start["uniform"]), 3), "heldout_psnr_end": round(psnr(end["uniform"]), 3),
           "peak_memory_gb": round(torch.cuda.max_memory_allocated(dev) / 1e9, 3),
           "model_and_state_gb": round((torch.cuda.max_memory_allocated(dev) - base_mem) / 1e9, 3),
           "ray_pool_gb": round(base_mem / 1e9, 3)}
    if net is not None:
        out["heldout_psnr_end_proposal_render"] = round(psnr(end["proposal"]), 3)
    if not quiet:
        print(json.dumps(out), flush=True)
    return (out, model, net) if return_state else out


def run_separable(a, data, quiet=False, return_state=False):
    """The training loop of ``run`` for the reference's separable model (SeparableRenderGrid):
    one fused forward + MSE + backward launch per step, then Adam on the layers and the
    offset and the fused Adam on the appearance grid."""
    if a.proposal or a.online_proposal or a.sh != 2 or a.storage != "f32" or a.save or a.resume:
        raise ValueError("--model separable trains the reference's fp32 SH-2 model with the uniform march only")
    dev = torch.device("cuda", torch.cuda.current_device())
    R = a.reso
    rays, origin, direction, target = data
    total = rays.shape[0]
    gen = torch.Generator(device=dev).manual_seed(a.seed + 1)
    held = torch.randint(0, total, (a.rays,), generator=gen, device=dev)
    torch.cuda.reset_peak_memory_stats(dev)
    base_mem = torch.cuda.memory_allocated(dev)
    model = fused.SeparableRenderGrid(R, a.k, a.interval, mode=a.mode, device=dev)
    layers = [model.xLayer, model.yLayer, model.zLayer, model.offset]
    opt_layers = torch.optim.Adam(layers, lr=a.lr)
    opt_grid = FusedGridAdam([model.renderData], lr=a.lr)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)

    def evaluate():
        with torch.no_grad():
            col = model(rays[held], origin[held], direction[held])
        return float(((col - target[held]) ** 2).mean())

    start = evaluate()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    log = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for step in range(1, a.steps + 1):
        idx = torch.randint(0, total, (a.rays,), generator=gen, device=dev)
        e0, e1, e2 = ev[step - 1]
        e0.record()
        loss.zero_()
        model.train_step(target[idx], rays[idx], origin[idx], direction[idx], loss=loss)
        e1.record()
        opt_grid.step()  # fused Adam on the appearance grid; zeroes its gradient
        opt_layers.step()
        opt_layers.zero_grad(set_to_none=True)
        e2.record()
        if not quiet and (step % a.log_every == 0 or step == a.steps):
            torch.cuda.synchronize()
            log.append({"step": step, "train_mse": float(loss) / (3 * a.rays),
                        "elapsed_s": round(time.perf_counter() - t0, 3)})
            print(json.dumps(log[-1]), flush=True)
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    render_ms = sum(x.elapsed_time(y) for x, y, _ in ev)
    opt_ms = sum(y.elapsed_time(z) for _, y, z in ev)
    end = evaluate()
    out = {"model": "separable (reference RenderGrid layers)", "reso": R, "steps": a.steps, "rays_per_step": a.rays,
           "lr": a.lr, "mode": a.mode, "k": a.k, "ms_per_step": round(1e3 * elapsed / a.steps, 3),
           "train_rays_per_s": round(a.steps * a.rays / elapsed), "render_ms": round(render_ms, 3),
           "optimizer_ms": round(opt_ms, 3), "render_rays_per_s": round(a.steps * a.rays / (render_ms / 1e3)),
           "heldout_psnr_start": round(psnr(start), 3), "heldout_psnr_end": round(psnr(end), 3),
           "peak_memory_gb": round(torch.cuda.max_memory_allocated(dev) / 1e9, 3),
           "model_and_state_gb": round((torch.cuda.max_memory_allocated(dev) - base_mem) / 1e9, 3)}
    if not quiet:
        print(json.dumps(out), flush=True)
    return (out, model, None) if return_state else out


def main(argv=None):
    return run(parser().parse_args(argv))


if __name__ == "__main__":
    main()
