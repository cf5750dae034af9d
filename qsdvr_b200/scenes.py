"""Seeded synthetic scenes, cameras and ray batches for tests and benchmarks.

The reference trains on nerf_synthetic (datasets/nerf_dataset.py); these builders stand
in for it with seeded scenes of the same shapes:

* ``sphere_grid``     dense 7-coefficient quadric grid of a sphere (exact per cell) plus
                      N(0, sigma) SDF noise;
* ``procedural_grid`` smooth union of 3 seeded spheres and a box, fitted per cell;
* ``appearance``      [(R+1)^3, 32] vertex data: SH DC ~ 0.5 + N(0, 0.05), higher orders
                      N(0, 0.1) (packed 9x3), diffuse U(0,1), metallic U(0,1), ao U(0.5,1);
* ``look_at``         OpenCV-convention pinhole cameras with the reference's cx = -W/2
                      (datasets/nerf_dataset.py:63-64) and row-major c2w rotation.

Cell (x, y, z) of an R^3 grid covers [(2x-R)/R, (2x+2-R)/R] on each axis; its local
coordinate u in [-1,1) maps to p = (u + k)/R with k = 2x + 1 - R (kernel/camera.cu:73-77).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .qsdvr import CameraArgs


# ----------------------------------------------------------------------------- cameras

def look_at(position, width: int, height: int, focal: float, near: float, far: float,
            target=(0.0, 0.0, 0.0), up=(0.0, 0.0, 1.0)) -> CameraArgs:
    """Pinhole camera at ``position`` looking at ``target`` (x right, y down, z forward)."""
    pos = np.asarray(position, np.float64)
    fwd = np.asarray(target, np.float64) - pos
    fwd /= np.linalg.norm(fwd)
    upv = np.asarray(up, np.float64)
    if abs(np.dot(fwd, upv)) > 0.999:
        upv = np.array([0.0, 1.0, 0.0])
    right = np.cross(fwd, upv)
    right /= np.linalg.norm(right)
    down = np.cross(fwd, right)
    rot = np.stack([right, down, fwd], 1)  # columns: camera axes in world space
    a = CameraArgs()
    a.width, a.height = int(width), int(height)
    a.rotation = rot.reshape(-1)
    a.translation = pos
    a.fx = a.fy = float(focal)
    a.cx = -width / 2.0
    a.cy = -height / 2.0
    a.near, a.far = float(near), float(far)
    a.pixelCount = a.width * a.height
    return a


def hemisphere_cameras(n: int, radius: float, width: int, height: int, focal: float, near: float, far: float,
                       seed: int = 0):
    """``n`` cameras uniform on the upper hemisphere of ``radius``, looking at the origin."""
    rng = np.random.default_rng(seed)
    cams = []
    for _ in range(n):
        z = rng.uniform(0.05, 1.0)
        phi = rng.uniform(0.0, 2 * math.pi)
        s = math.sqrt(1 - z * z)
        cams.append(look_at((radius * s * math.cos(phi), radius * s * math.sin(phi), radius * z), width, height,
                            focal, near, far))
    return cams


# ----------------------------------------------------------------------------- SDF grids

def _cell_k(R: int, device):
    return (2 * torch.arange(R, device=device, dtype=torch.float64) + 1 - R)


def sphere_grid(R: int, radius: float = 0.5, noise: float = 0.01, seed: int = 0, device="cpu") -> torch.Tensor:
    """[R,R,R,7] grid whose quadric in every cell is exactly |p|^2 - r^2 (scaled by R^2):
    a0..2 = 1, a3..5 = 2k, a6 = sum k^2 - R^2 r^2, then a6 += eps R |grad f(0)|, eps ~ N(0, noise),
    which shifts each cell's centre SDF by eps."""
    k = _cell_k(R, device)
    kz, ky, kx = torch.meshgrid(k, k, k, indexing="ij")
    g = torch.empty((R, R, R, 7), dtype=torch.float64, device=device)
    g[..., 0:3] = 1.0
    g[..., 3], g[..., 4], g[..., 5] = 2 * kx, 2 * ky, 2 * kz
    g[..., 6] = kx * kx + ky * ky + kz * kz - (R * radius) ** 2
    if noise:
        gen = torch.Generator(device=device).manual_seed(seed)
        eps = torch.randn((R, R, R), generator=gen, device=device, dtype=torch.float64) * noise
        grad0 = 2 * torch.sqrt(kx * kx + ky * ky + kz * kz).clamp_min(1.0)
        g[..., 6] += eps * R * grad0
    return g.float()


def _smin(a, b, k=0.1):
    h = torch.clamp(0.5 + 0.5 * (b - a) / k, 0.0, 1.0)
    return b * (1 - h) + a * h - k * h * (1 - h)


def procedural_sdf(p: torch.Tensor, seed: int = 0) -> torch.Tensor:
    """Smooth union of 3 seeded spheres (radii U(0.2,0.4)) and one box; p: [..., 3]."""
    rng = np.random.default_rng(seed)
    d = None
    for _ in range(3):
        c = torch.tensor(rng.uniform(-0.45, 0.45, 3), dtype=p.dtype, device=p.device)
        r = float(rng.uniform(0.2, 0.4))
        s = torch.linalg.norm(p - c, dim=-1) - r
        d = s if d is None else _smin(d, s)
    bc = torch.tensor(rng.uniform(-0.3, 0.3, 3), dtype=p.dtype, device=p.device)
    bh = torch.tensor(rng.uniform(0.15, 0.3, 3), dtype=p.dtype, device=p.device)
    q = torch.abs(p - bc) - bh
    box = torch.linalg.norm(torch.clamp(q, min=0.0), dim=-1) + torch.clamp(q.max(-1).values, max=0.0)
    return _smin(d, box)


def procedural_grid(R: int, seed: int = 0, device="cpu", chunk: int = 64) -> torch.Tensor:
    """[R,R,R,7] per-cell quadric fit of ``procedural_sdf`` around each cell centre c:
    a3..5 = grad sdf(c) / R, a0..2 = (1/2) d2 sdf/dx2 / R^2 (diagonal), a6 = sdf(c)."""
    k = _cell_k(R, device) / R
    out = torch.empty((R, R, R, 7), dtype=torch.float32, device=device)
    h = 0.5 / R
    for z0 in range(0, R, chunk):
        kz, ky, kx = torch.meshgrid(k[z0:z0 + chunk], k, k, indexing="ij")
        c = torch.stack([kx, ky, kz], -1)
        f0 = procedural_sdf(c, seed)
        out[z0:z0 + chunk, ..., 6] = f0.float()
        for ax in range(3):
            e = torch.zeros(3, dtype=c.dtype, device=device)
            e[ax] = h
            fp, fm = procedural_sdf(c + e, seed), procedural_sdf(c - e, seed)
            out[z0:z0 + chunk, ..., 3 + ax] = ((fp - fm) / (2 * h) / R).float()
            out[z0:z0 + chunk, ..., ax] = (0.5 * (fp - 2 * f0 + fm) / (h * h) / (R * R)).float()
    return out


# ----------------------------------------------------------------------------- appearance

def appearance(R: int, seed: int = 0, device="cpu", procedural: bool = False, sh_degree: int = 2) -> torch.Tensor:
    """[(R+1)^3, C] vertex data (vertex x + y(R+1) + z(R+1)^2), packed SH order.
    Degree 2: C = 32 (27 SH, diffuse 27..29, metallic 30, ao 31), the reference's layout;
    degree 3: C = 64 (48 SH, diffuse 48..50, metallic 51, ao 52, 53..63 zero)."""
    V = (R + 1) ** 3
    nsh = 3 * (sh_degree + 1) ** 2
    C = 32 if sh_degree == 2 else 64
    gen = torch.Generator(device=device).manual_seed(seed)
    d = torch.zeros((V, C), dtype=torch.float32, device=device)
    d[:, 0:3] = 0.5 + 0.05 * torch.randn((V, 3), generator=gen, device=device)
    d[:, 3:nsh] = 0.1 * torch.randn((V, nsh - 3), generator=gen, device=device)
    d[:, nsh:nsh + 3] = torch.rand((V, 3), generator=gen, device=device)
    d[:, nsh + 3] = torch.rand(V, generator=gen, device=device)
    d[:, nsh + 4] = 0.5 + 0.5 * torch.rand(V, generator=gen, device=device)
    if procedural:
        # smooth seeded RGB field projected onto the DC coefficient and the diffuse colour
        n = torch.arange(R + 1, device=device, dtype=torch.float32) * (2.0 / R) - 1.0
        rng = np.random.default_rng(seed + 17)
        f = torch.tensor(rng.uniform(1.0, 4.0, (3, 3)), dtype=torch.float32, device=device)
        ph = torch.tensor(rng.uniform(0, 2 * math.pi, 3), dtype=torch.float32, device=device)
        for z0 in range(0, R + 1, 32):
            zz, yy, xx = torch.meshgrid(n[z0:z0 + 32], n, n, indexing="ij")
            p = torch.stack([xx, yy, zz], -1).reshape(-1, 3)
            rgb = 0.5 + 0.45 * torch.sin(p @ f.T + ph)
            lo, hi = z0 * (R + 1) ** 2, min(R + 1, z0 + 32) * (R + 1) ** 2
            d[lo:hi, 0:3] = rgb / (2 * 0.28209479177387814)
            d[lo:hi, nsh:nsh + 3] = rgb
    return d
