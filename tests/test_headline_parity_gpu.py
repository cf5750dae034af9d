"""Parity at the headline configuration, entry by entry.

The bench's own plain256 batch (256^3 quadric grid, [(257)^3, 32] appearance grid, fp32,
compat mode, 65,536 random rays from 100 seeded 800^2 views, 256 samples/ray, k = 5) goes
through the fused train kernel exactly as the bench runs it, with the rays taken in the
Morton order of their midpoints (``fused.ray_order``).  The reference build
(oracle/_ref, the unmodified kernel/*.cu) runs its own op chain on the same batch
(models/render.py:225-234 forward, MSE gradient, the Functions' backwards).

Bars:
* image within 1e-5 absolute;
* both gradients within 1e-4 norm-wise (max |a - b| / max |b|);
* entry by entry, against the exact gradient (the float64 oracle on the same batch, on the
  host, in chunks of rays): on every finite entry above 1e-3 of the largest, the fused kernel's
  relative error is at most twice the reference build's own worst error there, and its
  0.999 quantile at most twice the reference's.  Both accumulate sums of many contributions
  of mixed sign with float atomics in an arbitrary order, so the reference itself is not
  within 1e-4 of the exact value on every such entry; the kernel against the reference is
  printed beside it;
* the same batch in bf16 storage with the appearance gradient accumulated in bf16
  (``bf16g_256``): that gradient within 2e-2 norm-wise of the fp32-accumulated one, the
  colours identical and the SDF gradient within 1e-5.
The measured errors are printed (pytest -s)."""
import json

import numpy as np
import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _entrywise(ours, ref, floor=1e-3):
    """Largest |ours - ref| / |ref| over the finite entries with |ref| > floor * max |ref|, their
    count, the 0.999 quantile of that error, and the count of non-finite reference entries
    (rel_err requires ours to be non-finite at exactly those)."""
    a = ours.double().reshape(-1)
    b = ref.double().reshape(-1)
    fin = torch.isfinite(b)
    big = fin & (b.abs() > floor * b[fin].abs().max())
    rel = (a[big] - b[big]).abs() / b[big].abs()
    q = float(torch.sort(rel).values[int(0.999 * (rel.numel() - 1))]) if rel.numel() else 0.0
    return float(rel.max()) if rel.numel() else 0.0, int(big.sum()), q, int((~fin).sum())


def oracle_gradients_f64(grid7, data, inp, target, k, chunk=8192):
    """The MSE gradients (mean over all rays and channels) of both grids by the float64 oracle
    on the host, in chunks of rays: each chunk's sample lists are contiguous (packed offsets),
    so it is rendered on its own with the loss scaled by the whole batch, and the chunks'
    gradients add up."""
    import oracle.oracle as O

    rays = inp["rayList"].cpu().long()
    n = rays.shape[0]
    g7 = grid7.detach().double().cpu()
    dd = data.detach().double().cpu()
    tgt = target.detach().double().cpu()
    lists = {kk: v.cpu() for kk, v in inp.items() if kk != "rayList"}
    gg = torch.zeros_like(g7)
    gd = torch.zeros_like(dd)
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        sub = rays[a:b].clone()
        s0, m0 = int(sub[0, 1]), int(sub[0, 3])
        s1 = int((sub[:, 1] + sub[:, 0]).max())
        m1 = int((sub[:, 3] + sub[:, 2]).max())
        sub[:, 1] -= s0
        sub[:, 3] -= m0
        part = {"rayList": sub}
        for kk in ("sdfPointList", "sdfIndexList"):
            part[kk] = lists[kk][s0:s1]
        for kk in ("renderPointList", "renderIndexList", "viewDirList"):
            part[kk] = lists[kk][m0:m1]
        g = g7.requires_grad_()
        d = dd.requires_grad_()
        img = O.render(g, d, part, k, compat=True)
        loss = ((img - tgt[a:b]) ** 2).sum() / (3.0 * n)
        dg7, ddd = torch.autograd.grad(loss, (g, d))
        gg += dg7
        gd += ddd
        del dg7, ddd, img, loss
    return gg, gd


def test_headline_batch_entrywise_parity_with_reference():
    import bench
    from oracle.build_ref import load_reference
    from qsdvr_b200 import fused, qsdvr
    from tests.golden.make_golden import reference_render

    ref = load_reference()
    if ref is None:
        pytest.skip("reference build absent")
    cfg = dict(bench.WORKLOADS["plain256"])
    R, k, interval = cfg["R"], bench.K_LOGISTIC, cfg["interval"]
    scene = bench.build_scene(cfg, DEV, seed=0)
    batch = bench.make_batches(scene, cfg, 1, DEV, seed=1000)[0]
    del scene["gt"]
    sdf, data = scene["model"]
    rays, origin, direction, target = batch["rays"], batch["origin"], batch["dir"], batch["target"]
    order = fused.ray_order(rays, origin, direction, interval)

    sg, dg = torch.zeros_like(sdf), torch.zeros_like(data)
    col, _ = fused.render_train(target, rays, origin, direction, sdf, data, R, interval, k, sg, dg, mode="compat",
                                order=order)

    # the reference's chain on sample lists of the same rays (compact offsets; the lists are
    # bit-exact with the reference's own GenerateRayPoints)
    r = rays.clone()
    ns = r[:, 0].long()
    nr = torch.clamp(ns - 1, min=0)
    r[:, 1] = (torch.cumsum(ns, 0) - ns).int()
    r[:, 2] = nr.int()
    r[:, 3] = (torch.cumsum(nr, 0) - nr).int()
    S, M = int(ns.sum()), int(nr.sum())
    inp = dict(sdfPointList=torch.empty((S, 3), device=DEV), sdfIndexList=torch.empty(S, dtype=torch.int32, device=DEV),
               renderPointList=torch.empty((M, 3), device=DEV),
               renderIndexList=torch.empty(M, dtype=torch.int32, device=DEV), viewDirList=torch.empty((M, 3), device=DEV))
    qsdvr.GenerateRayPoints(None, inp["sdfPointList"], inp["sdfIndexList"], inp["renderPointList"],
                            inp["renderIndexList"], inp["viewDirList"], r, origin, direction, interval, R)
    inp["rayList"] = r
    grid7 = sdf[:, :7].contiguous()
    img, g7, gd = reference_render(ref, grid7, data, inp, R, k, target)
    # the exact gradient: the float64 oracle (compat: the reference's formulas) on the host
    gg64, gd64 = oracle_gradients_f64(grid7, data, inp, target, k)
    gg64, gd64 = gg64.to(DEV), gd64.to(DEV)
    del inp
    torch.cuda.empty_cache()

    e_img = float((col - img).abs().max())
    e_sdf, e_data = rel_err(sg[:, :7].cpu(), g7.cpu()), rel_err(dg.cpu(), gd.cpu())
    w_sdf, n_sdf, q_sdf, nf_sdf = _entrywise(sg[:, :7], g7)
    w_data, n_data, q_data, nf_data = _entrywise(dg, gd)
    fin_s = torch.isfinite(g7) & torch.isfinite(gg64)  # the reference's Q10 entries aside
    x_sdf = _entrywise(sg[:, :7][fin_s], gg64[fin_s])  # ours vs exact
    r_sdf = _entrywise(g7[fin_s], gg64[fin_s])         # the reference vs exact
    x_data = _entrywise(dg, gd64)
    r_data = _entrywise(gd, gd64)

    # bf16 storage, appearance gradient accumulated in fp32 and in bf16 (bf16g_256)
    s16, d16 = fused.sdf_cells_bf16(sdf), data.to(torch.bfloat16)
    out = {}
    for gdt in (torch.float32, torch.bfloat16):
        sgb = torch.zeros_like(sdf)
        dgb = torch.zeros(data.shape, dtype=gdt, device=DEV)
        cb, _ = fused.render_train(target, rays, origin, direction, s16, d16, R, interval, k, sgb, dgb, mode="compat",
                                   transmittance="log", order=order)
        out[gdt] = (cb, sgb, dgb)
    c32, s32, d32 = out[torch.float32]
    c16, s16g, d16g = out[torch.bfloat16]
    e_bf16g = rel_err(d16g.float().cpu(), d32.cpu())
    e_bf16_sdf = rel_err(s16g.cpu(), s32.cpu())
    print("\n" + json.dumps({
        "workload": "plain256 bench batch: 65536 rays, Morton ray order, compat fp32", "render_samples": M,
        "image_max_abs": e_img, "sdf_grad_normwise": e_sdf, "data_grad_normwise": e_data,
        "sdf_grad_entrywise_max": w_sdf, "sdf_entries_checked": n_sdf, "sdf_entrywise_q999": q_sdf,
        "data_grad_entrywise_max": w_data, "data_entries_checked": n_data, "data_entrywise_q999": q_data,
        "nonfinite_reference_entries": [nf_sdf, nf_data],
        "vs_float64": {"sdf": {"ours_max": x_sdf[0], "reference_max": r_sdf[0], "ours_q999": x_sdf[2],
                               "reference_q999": r_sdf[2], "entries": x_sdf[1]},
                       "data": {"ours_max": x_data[0], "reference_max": r_data[0], "ours_q999": x_data[2],
                                "reference_q999": r_data[2], "entries": x_data[1]}},
        "bf16g_data_grad_normwise_vs_fp32_accumulation": e_bf16g, "bf16g_sdf_grad_vs_fp32": e_bf16_sdf}))
    assert e_img < 1e-5
    assert e_sdf < 1e-4 and e_data < 1e-4
    for ours, theirs in ((x_sdf, r_sdf), (x_data, r_data)):
        assert ours[1] > 1000
        assert ours[0] <= 2 * theirs[0] and ours[2] <= 2 * theirs[2]
    assert torch.equal(c32, c16)
    assert 0 < e_bf16g < 2e-2 and e_bf16_sdf < 1e-5
    assert np.isfinite([e_img, e_sdf, e_data, w_sdf, w_data, x_sdf[0], x_data[0]]).all()
