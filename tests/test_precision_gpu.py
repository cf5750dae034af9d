"""The precision form against the float64 oracle, side by side with the fp32 plain path.

Both storage forms render the same model, the FP32 master grids of the seeded procedural
scene, and both are compared with the float64 oracle evaluated on those masters (image, and
the MSE gradients of both grids; errors norm-wise: max |a - b| / max |b|).

The procedural scene's quadric fit has cells where |grad f| is small against f (along the
medial surfaces of its box); there the SDF sample f / |grad f| / R cancels badly in any
float32 arithmetic, and the same formulas evaluated by torch in float32 miss the float64
gradient of those coefficients by tens of percent.  The SDF-gradient bars therefore apply
where float32 arithmetic itself can be right: entries on which the float32 torch oracle agrees
with the float64 one within 1e-4 of the largest entry (the count left out is printed).

Bars: fp32 plain path — image within 1e-5 absolute, gradients within 1e-4 (the parity bars).
BF16 form (bf16 grids read by the kernel, fp32 arithmetic, compensated log-transmittance).
Its error is the storage rounding, and for the SDF-coefficient gradient that rounding meets
a discontinuity: the NeuS alpha max((E1 - E0) / (1 + E1), 0) (kernel/render.cu:244) switches a
sample between active and inactive where the SDF barely changes along the ray, and each such
switch moves that sample's SDF gradient by its own size.  float32 arithmetic alone, on the
fp32 masters, already moves the SDF gradient by ~1.2e-2 in L2 norm on this scene (0.22
max-abs) through those switches.  A plain bf16 rounding of the cells rescales each cell's SDF
by up to 2^-9 (the rounding of |grad f| through a3..a5), ~1e-3 of absolute SDF away from the
surface, and gave 0.40 in L2 (0.76 max-abs).  The stored cells therefore keep a6 compensated
for that rescaling and split into two bf16 (qsdvr_sdf_cells_bf16): the L2 error falls to
~4.5e-2 (SH 2) / ~4.9e-2 (SH 3), within 4x of float32 arithmetic.  Bars: image 2e-3 absolute,
appearance gradient 1e-2, SDF-coefficient gradient 7e-2 in L2 and 0.45 max-abs (all entries),
and at most a quarter of the plain rounding's L2 error, which the test measures beside it.
The measured errors are printed (pytest -s)."""
import numpy as np
import pytest
import torch

import oracle.oracle as O

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _oracle(grid7, data, inp, target, k, sh, dtype):
    """Image and MSE gradients of the oracle with its arithmetic in ``dtype``."""
    saved = O.DTYPE
    O.DTYPE = dtype
    try:
        g7 = grid7.to(dtype).requires_grad_()
        dd = data.to(dtype).requires_grad_()
        img = O.render(g7, dd, inp, k, compat=False, sh_degree=sh)
        loss = ((img - target.to(dtype)) ** 2).mean()
        gg, gd = torch.autograd.grad(loss, (g7, dd))
    finally:
        O.DTYPE = saved
    return img.detach().double(), gg.double(), gd.double()


def _err(a, b, mask=None):
    a, b = a.double().reshape(b.shape), b.double()
    if mask is not None:
        a, b = a[mask], b[mask]
    return float((a - b).abs().max() / b.abs().max())


@pytest.mark.parametrize("sh", [2, 3])
def test_precision_form_error_vs_oracle(sh):
    from qsdvr_b200 import _lib, fused, scenes
    from qsdvr_b200.camera import Camera

    _lib.lib()
    R, k, interval, size = 64, 5.0, 4.0 / 256, 64
    a = scenes.hemisphere_cameras(1, 4.03, size, size, 1111.1 * size / 800, 2.0, 6.0, seed=0)[0]
    cam = Camera(a, interval, R)
    cam.GenerateRayPoints(torch.ones(size * size, dtype=torch.bool))
    grid8 = fused.pad_grid7(scenes.procedural_grid(R, seed=0).reshape(-1, 7)).to(DEV)
    data = scenes.appearance(R, seed=0, procedural=True, sh_degree=sh).to(DEV)
    n = cam.rayList.shape[0]
    target = torch.rand((n, 3), generator=torch.Generator().manual_seed(1)).to(DEV)

    pts = cam.GetRayPoints()
    inp = {kk: v.cpu() for kk, v in pts.items() if kk != "rayList"}
    inp["rayList"] = pts["rayList"].cpu().long()
    g7, dcpu, tcpu = grid8[:, :7].cpu(), data.cpu(), target.cpu()
    img64, gg64, gd64 = _oracle(g7, dcpu, inp, tcpu, k, sh, torch.float64)
    _, gg32, _ = _oracle(g7, dcpu, inp, tcpu, k, sh, torch.float32)
    ok = (gg32 - gg64).abs() <= 1e-4 * gg64.abs().max()  # where float32 arithmetic can be right

    errs = {}
    forms = {"f32": (grid8, data), "bf16": (fused.sdf_cells_bf16(grid8), data.to(torch.bfloat16)),
             "bf16-plain": (grid8.to(torch.bfloat16), data.to(torch.bfloat16))}
    for storage, (g, d) in forms.items():
        sg, dg = torch.zeros_like(grid8), torch.zeros_like(data)
        img, _ = fused.render_train(target, cam.rayList, cam.originList, cam.dirList, g, d, R, interval, k, sg, dg,
                                    mode="fixed", transmittance="product" if storage == "f32" else "log")
        diff = (img.cpu().double() - img64).abs()
        sgc = sg[:, :7].cpu()
        errs[storage] = dict(image_max=float(diff.max()), image_mean=float(diff.mean()),
                             sdf_grad=_err(sgc, gg64, ok), sdf_grad_all=_err(sgc, gg64),
                             sdf_grad_l2=float((sgc.double() - gg64).norm() / gg64.norm()),
                             data_grad=_err(dg.cpu(), gd64))
    l2_32 = float((gg32 - gg64).norm() / gg64.norm())
    print(f"\nSH degree {sh}, R={R}, {n} rays, k={k}: error vs the float64 oracle on the fp32 masters "
          f"({int((~ok).sum())} of {ok.numel()} SDF-gradient entries ill-conditioned in float32; "
          f"float32 torch oracle: SDF grad {_err(gg32, gg64):.3e} max-abs, {l2_32:.3e} L2)")
    for storage, e in errs.items():
        print(f"  {storage:10s} image max {e['image_max']:.3e} mean {e['image_mean']:.3e}  grad: sdf "
              f"{e['sdf_grad']:.3e} (all entries {e['sdf_grad_all']:.3e}, L2 {e['sdf_grad_l2']:.3e}), "
              f"data {e['data_grad']:.3e}")
    f, b, bp = errs["f32"], errs["bf16"], errs["bf16-plain"]
    assert int((~ok).sum()) < 1e-4 * ok.numel()
    assert f["image_max"] < 1e-5 and f["sdf_grad"] < 1e-4 and f["data_grad"] < 1e-4
    assert b["image_max"] < 2e-3 and b["data_grad"] < 1e-2
    assert b["sdf_grad_all"] < 0.45 and b["sdf_grad_l2"] < 7e-2
    assert b["sdf_grad_l2"] < 0.25 * bp["sdf_grad_l2"]
    # the BF16 form's error is the storage rounding, well above the fp32 arithmetic's
    assert b["image_max"] > 10 * f["image_max"]
    assert np.isfinite([v for e in errs.values() for v in e.values()]).all()
