"""Speed of the reference's own CUDA path (built from its sources into oracle/_ref) against
the fused kernel, on the same 256^3 training batch.

The reference's training step (test.py:26-35 with models/render.py:225-234) runs, on sample
lists that its dataset precomputes per batch (datasets/utils.py:17-33): SampleSDF,
SampleNormal, GridInterpolation, Shader and RayAggregate forward, then their backward ops,
each Function's backward allocating zeroed dense gradient grids (models/render.py:28-33,
136-146, 160-169).  Timed here: exactly that chain (forward + MSE gradient + backward, with
the dense zero-fills), against zero-fill + one fused train launch, and against the same op
chain run through this library's drop-in ``qsdvr`` module (same function names and
arguments, this library's per-op kernels).  All three see identical rays, grids and
targets; the reference's colours and gradients are checked against both of ours so the timed
computations are the same work.  Prints one JSON line."""
import json

import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _time(fn, reps=5):
    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def test_fused_train_faster_than_reference_chain():
    from oracle.build_ref import load_reference
    from qsdvr_b200 import fused, scenes
    from qsdvr_b200.camera import Camera
    from tests.golden.make_golden import reference_render

    ref = load_reference()
    if ref is None:
        pytest.skip("reference build absent")
    R, k, interval, n_rays = 256, 5.0, 4.0 / 256, 65536
    cams = scenes.hemisphere_cameras(4, 4.03, 800, 800, 1111.1, 2.0, 6.0, seed=0)
    rays, origin, direction = [], [], []
    for a in cams:
        c = Camera(a, interval, R, device=DEV)
        c.GenerateRayPoints(torch.ones(800 * 800, dtype=torch.bool))
        rays.append(c.rayList)
        origin.append(c.originList)
        direction.append(c.dirList)
    rays, origin, direction = torch.cat(rays), torch.cat(origin), torch.cat(direction)
    idx = torch.randint(0, rays.shape[0], (n_rays,), generator=torch.Generator(device=DEV).manual_seed(1),
                        device=DEV)
    # one batch with compact sample offsets, and its sample lists (the dataset's
    # precomputation; GenerateRayPoints is bit-exact with the reference's)
    r = rays[idx].clone()
    ns = r[:, 0].long()
    nr = torch.clamp(ns - 1, min=0)
    r[:, 1] = (torch.cumsum(ns, 0) - ns).int()
    r[:, 2] = nr.int()
    r[:, 3] = (torch.cumsum(nr, 0) - nr).int()
    o, d = origin[idx].contiguous(), direction[idx].contiguous()
    S, M = int(ns.sum()), int(nr.sum())
    inp = dict(sdfPointList=torch.empty((S, 3), device=DEV), sdfIndexList=torch.empty(S, dtype=torch.int32, device=DEV),
               renderPointList=torch.empty((M, 3), device=DEV),
               renderIndexList=torch.empty(M, dtype=torch.int32, device=DEV), viewDirList=torch.empty((M, 3), device=DEV))
    from qsdvr_b200 import qsdvr

    qsdvr.GenerateRayPoints(None, inp["sdfPointList"], inp["sdfIndexList"], inp["renderPointList"],
                            inp["renderIndexList"], inp["viewDirList"], r, o, d, interval, R)
    inp["rayList"] = r
    grid7 = scenes.sphere_grid(R, 0.5, 0.01, seed=0, device=DEV).reshape(-1, 7).contiguous()
    data = scenes.appearance(R, seed=1, device=DEV)
    target = torch.rand((n_rays, 3), generator=torch.Generator(device=DEV).manual_seed(2), device=DEV)
    grid8 = fused.pad_grid7(grid7)
    sg, dg = torch.zeros_like(grid8), torch.zeros_like(data)

    def ours():
        sg.zero_()
        dg.zero_()
        fused.render_train(target, r, o, d, grid8, data, R, interval, k, sg, dg)

    ref_ms = _time(lambda: reference_render(ref, grid7, data, inp, R, k, target))
    our_ms = _time(ours)
    dropin_ms = _time(lambda: reference_render(qsdvr, grid7, data, inp, R, k, target))
    img2, g72, gd2 = reference_render(qsdvr, grid7, data, inp, R, k, target)
    img, g7, gd = reference_render(ref, grid7, data, inp, R, k, target)
    ours()
    col = fused.render_forward(r, o, d, grid8, data, R, interval, k)
    torch.cuda.synchronize()
    assert (col - img).abs().max().item() < 1e-5
    assert rel_err(sg[:, :7].cpu(), g7.cpu()) < 1e-4 and rel_err(dg.cpu(), gd.cpu()) < 1e-4
    assert (img2 - img).abs().max().item() < 1e-5
    assert rel_err(g72.cpu(), g7.cpu()) < 1e-4 and rel_err(gd2.cpu(), gd.cpu()) < 1e-4
    print(json.dumps({"workload": "R=256 fp32 compat, 65536 rays from 800^2 views, 256 samples/ray",
                      "render_samples": M, "reference_cuda_ms": round(ref_ms, 3), "fused_ms": round(our_ms, 3),
                      "reference_rays_per_s": round(n_rays / ref_ms * 1e3), "fused_rays_per_s":
                      round(n_rays / our_ms * 1e3), "speedup": round(ref_ms / our_ms, 2),
                      "dropin_op_chain_ms": round(dropin_ms, 3), "dropin_speedup": round(ref_ms / dropin_ms, 2)}))
    assert our_ms < ref_ms
