"""ORACLE / CPU baseline — the reference's pure-torch render path on the host.

Test and benchmark infrastructure only (imported by tests/ and by bench.py's CPU-baseline
leg).  Restates models/render_torch.py:117-168 (RenderGridTorch.forward) so it runs on
device="cpu" and is differentiable with torch autograd, keeping its structure: vectorised
quadric sampling (models/render_torch.py:77-100), trilinear fetch (:128-143), shader
(:144-152, packed SH reshape (-1, 9, 3), truncated SH constants :175-179) and the per-ray
Python compositing loop (:155-166).  Two reference bugs are fixed so the output means
something: every ray writes its own image row (the reference writes image[0], :167), and
the sample cell index addresses the vertex grid with stride R+1 neighbours exactly as
the CUDA path does (the reference's torch path uses stride R, :128-131).  The SDF is a
dense [R^3,7] quadric grid (the grid QuadricGridTorch.forward builds, :65-76).
"""
from __future__ import annotations

import torch

# models/render_torch.py:175-179 (truncated constants, as in the reference's torch path)
SH_FACTOR_TORCH = (0.2820947917, 0.4886025119, 0.4886025119, 0.4886025119, 1.0925484305, 1.0925484305, 0.3153915652,
                   1.0925484305, 0.5462742152)


def _lerp(a, b, c):  # models/render_torch.py:170-172
    c = c.reshape([-1, 1])
    return (1 - c) * a + b * c


def _sh(v, coef):  # models/render_torch.py:174-195
    f = SH_FACTOR_TORCH
    x4 = v[:, 0:1] * v[:, 2:3]
    zz = v[:, 2:3] * v[:, 2:3]
    xx = v[:, 0:1] * v[:, 0:1]
    x5 = v[:, 0:1] * v[:, 1:2]
    x6 = 2.0 * v[:, 1:2] * v[:, 1:2] - zz - xx
    x7 = v[:, 1:2] * v[:, 2:3]
    x8 = zz - xx
    return (f[0] * coef[:, 0, :] + f[1] * coef[:, 1, :] * v[:, 0:1] + f[2] * coef[:, 2, :] * v[:, 1:2] +
            f[3] * coef[:, 3, :] * v[:, 2:3] + f[4] * coef[:, 4, :] * x4 + f[5] * coef[:, 5, :] * x5 +
            f[6] * coef[:, 6, :] * x6 + f[7] * coef[:, 7, :] * x7 + f[8] * coef[:, 8, :] * x8)


def render_torch_cpu(sdf_grid7: torch.Tensor, render_data: torch.Tensor, inp: dict, reso: int, k: float):
    """RenderGridTorch.forward on the CPU.  sdf_grid7: [R^3*7] or [R^3,7]; render_data:
    [(R+1)^3, 32]; inp: the GenerateRayPoints dict (CPU tensors).  Returns [N,3]."""
    grid = sdf_grid7.reshape(-1)
    si = inp["sdfIndexList"].long()
    sp = inp["sdfPointList"]
    index = si * 7
    a0 = grid[index] * sp[:, 0]
    a1 = grid[index + 1] * sp[:, 1]
    a2 = grid[index + 2] * sp[:, 2]
    a3, a4, a5, a6 = grid[index + 3], grid[index + 4], grid[index + 5], grid[index + 6]
    sdf = ((a0 + a3) * sp[:, 0] + (a1 + a4) * sp[:, 1] + (a2 + a5) * sp[:, 2] + a6) / torch.sqrt(
        (2 * a0 + a3) * (2 * a0 + a3) + (2 * a1 + a4) * (2 * a1 + a4) + (2 * a2 + a5) * (2 * a2 + a5)) / reso
    ri = inp["renderIndexList"].long()
    rp = inp["renderPointList"]
    index = ri * 7
    n = torch.cat([2 * grid[index] * rp[:, 0] + grid[index + 3], 2 * grid[index + 1] * rp[:, 1] + grid[index + 4],
                   2 * grid[index + 2] * rp[:, 2] + grid[index + 5]]).reshape(3, -1).transpose(0, 1)
    normal = torch.nn.functional.normalize(n)
    R1 = reso + 1
    i000 = ri
    i010 = i000 + R1
    i100 = i000 + R1 * R1
    i110 = i100 + R1
    d = render_data
    p = (rp + 1) / 2
    a00 = _lerp(d[i000, :], d[i000 + 1, :], p[:, 0])
    a01 = _lerp(d[i010, :], d[i010 + 1, :], p[:, 0])
    b0 = _lerp(a00, a01, p[:, 1])
    a10 = _lerp(d[i100, :], d[i100 + 1, :], p[:, 0])
    a11 = _lerp(d[i110, :], d[i110 + 1, :], p[:, 0])
    b1 = _lerp(a10, a11, p[:, 1])
    data = _lerp(b0, b1, p[:, 2])
    ao, diffuse, metallic = data[:, 31:32], data[:, 27:30], data[:, 30:31]
    specular = data[:, :27].reshape((-1, 9, 3))
    view = inp["viewDirList"]
    vdotn = (view * normal).sum(dim=1).reshape((-1, 1))
    reflect = view - normal * (2.0 * vdotn)
    color = diffuse * (1 - metallic) + _sh(reflect, specular) * metallic
    rgb = color * ao
    rays = inp["rayList"].tolist()
    rows = []
    for info in rays:  # models/render_torch.py:155-167, one row per ray
        if info[0] == 0:
            rows.append(torch.zeros(3, dtype=rgb.dtype))
            continue
        e_i = torch.exp(-k * sdf[info[1]])
        T = torch.ones((), dtype=rgb.dtype)
        c = torch.zeros(3, dtype=rgb.dtype)
        for i in range(info[2]):
            e_i1 = torch.exp(-k * sdf[info[1] + i + 1])
            alpha = torch.clamp((e_i1 - e_i) / (1.0 + e_i1), 0.0, 10.0)
            c = c + rgb[info[3] + i] * alpha * T
            e_i = e_i1
            T = T * (1 - alpha)
        rows.append(c)
    return torch.stack(rows)
