"""Differentiation form: the fused backward against central finite differences of an FP64
forward on the GPU (48^3 grid, 1024 seeded rays, h = 1e-3, 256 SDF + 256 SH entries)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = "cuda"


def test_fused_backward_matches_fp64_finite_differences():
    from qsdvr_b200 import fused, gradcheck, scenes
    from qsdvr_b200.camera import Camera

    R, k, interval = 48, 8.0, 4.0 / 128
    # 1024 rays: a 32 x 32 camera looking at a noisy sphere
    args = scenes.look_at((1.3, -3.6, 1.1), 32, 32, 45.0, 2.0, 6.0)
    cam = Camera(args, interval, R)
    cam.GenerateRayPoints(torch.ones(32 * 32, dtype=torch.bool))
    rays, origin, direction = cam.rayList, cam.originList, cam.dirList
    assert rays.shape[0] == 1024
    grid = fused.pad_grid7(scenes.sphere_grid(R, 0.5, 0.01, seed=11).reshape(-1, 7)).to(DEV)
    data = scenes.appearance(R, seed=11).to(DEV)
    target = torch.rand((1024, 3), generator=torch.Generator().manual_seed(12)).to(DEV)
    sg, dg = torch.zeros_like(grid), torch.zeros_like(data)
    fused.render_train(target, rays, origin, direction, grid, data, R, interval, k, sg, dg, mode="fixed")
    # 256 SDF coefficients and 256 SH coefficients among the entries the rays touch
    gen = torch.Generator().manual_seed(13)
    sdf_touched = torch.nonzero(sg.view(-1)[:R ** 3 * 8].cpu() != 0).view(-1)
    sdf_touched = sdf_touched[(sdf_touched % 8) < 7]
    sh_mask = torch.zeros(32, dtype=torch.bool)
    sh_mask[:27] = True
    dflat = dg.view(-1).cpu()
    sh_touched = torch.nonzero((dflat != 0) & sh_mask.repeat(dflat.numel() // 32)).view(-1)
    se = sdf_touched[torch.randperm(sdf_touched.numel(), generator=gen)[:256]]
    de = sh_touched[torch.randperm(sh_touched.numel(), generator=gen)[:256]]
    fd_s, fd_d = gradcheck.finite_differences(rays, origin, direction, grid, data, R, interval, k, target, se, de)
    g_s = sg.view(-1)[se.to(DEV)].double().cpu()
    g_d = dg.view(-1)[de.to(DEV)].double().cpu()
    for name, fd, g in (("sdf", fd_s, g_s), ("sh", fd_d, g_d)):
        scale = float(fd.abs().max())
        rel = (fd - g).abs() / torch.clamp(fd.abs(), min=1e-2 * scale)
        normwise = float((fd - g).norm() / fd.norm())
        print(f"{name}: entries {len(fd)}, norm-wise rel err {normwise:.2e}, median {float(rel.median()):.2e}, "
              f"95% {float(np.quantile(rel.numpy(), 0.95)):.2e}, max {float(rel.max()):.2e}")
        assert normwise < 1e-3, name
        assert float(np.quantile(rel.numpy(), 0.95)) < 1e-2, name
