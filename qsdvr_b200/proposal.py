"""Proposal network: 64 coarse MLP evaluations + 32 fine samples per ray in place of the
uniform march (no counterpart in the reference).

``ProposalNet`` holds the MLP (fp32 master parameters, the bf16 copy the tensor-core kernels
read, Adam state).  It is trained online on the renderer's own per-sample opacities: a
uniform-march forward writes the alpha of every render sample, ``targets`` turns them into
(position, density) pairs and ``train_step`` fits the density bound.  ``sample`` gives each
ray its 33 fine SDF positions; ``render`` renders with them (32 render samples per ray).
The uniform march stays the fallback (an untrained network) and the reference its PSNR is
measured against.
"""
from __future__ import annotations

import ctypes
import math

import torch

from . import _lib, fused
from ._lib import F32, P, U32, U64, call
from .optim import adam_step

N_PARAMS = 6280
N_COARSE = 64
N_FINE_T = 33

_lib.extra_signatures({
    "qsdvr_mlp_density": [P, U32, P, P, P, U32, F32, P, P, P],
    "qsdvr_mlp_train": [P, U32, P, F32, P, P, P],
    "qsdvr_proposal_sample": [P, U32, F32, F32, P, P, P],
    "qsdvr_proposal_targets": [P, P, P, U32, F32, P, U64, P, P],
    "qsdvr_proposal_draw": [P, P, P, U32, F32, P, U64, U32, U32, P, P],
    "qsdvr_mlp_launch_shape": [ctypes.c_int, U32, P, P],
    "qsdvr_check_bounded_wait": [U64, P, P],
})

INFER_MIX = 0.05  # uniform share of the fine-sample pdf when rendering
TRAIN_MIX = 0.25  # and when training the grid at the proposal's samples


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream(dev):
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def init_params(seed: int = 0, device="cuda") -> torch.Tensor:
    """Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights, zero biases (b3 = 0: bound 0.69)."""
    gen = torch.Generator().manual_seed(seed)
    w = torch.zeros(N_PARAMS, dtype=torch.float32)
    w[:2048] = (torch.rand(2048, generator=gen) * 2 - 1) / math.sqrt(28)
    w.view(-1)[:2048].view(64, 32)[:, 28:] = 0.0  # encoding features 28..31 are always zero
    w[2048:6144] = (torch.rand(4096, generator=gen) * 2 - 1) / math.sqrt(64)
    w[6208:6272] = (torch.rand(64, generator=gen) * 2 - 1) / math.sqrt(64)
    return w.to(device)


class ProposalNet:
    """The density-bound MLP with its optimizer state."""

    def __init__(self, device="cuda", seed: int = 0, lr: float = 5e-3, under_weight: float = 4.0):
        self.device = torch.device(device)
        self.params = init_params(seed, self.device)
        self.params_bf16 = self.params.to(torch.bfloat16)
        self.grad = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        self.step_count = 0
        self.lr = lr
        self.under_weight = under_weight
        self._bufs: dict = {}

    # ---- inference
    def density(self, points: torch.Tensor) -> torch.Tensor:
        """Density bound at points [P,3] or [P,4] (float32)."""
        pts = points.float()
        if pts.shape[1] == 3:
            pts = torch.cat([pts, torch.zeros_like(pts[:, :1])], 1)
        pts = pts.contiguous()
        out = torch.empty(pts.shape[0], dtype=torch.float32, device=self.device)
        call("qsdvr_mlp_density", _p(pts), pts.shape[0], None, None, None, 0, 0.0, _p(self.params_bf16), _p(out),
             _stream(self.device))
        return out

    def coarse_density(self, rays, origin, direction, interval) -> torch.Tensor:
        """[N, 64] density bound at the coarse points of every ray."""
        n = rays.shape[0]
        out = torch.empty((n, N_COARSE), dtype=torch.float32, device=self.device)
        call("qsdvr_mlp_density", None, 0, _p(rays), _p(origin), _p(direction), n, float(interval),
             _p(self.params_bf16), _p(out), _stream(self.device))
        return out

    def sample(self, rays, origin, direction, interval, uniform_mix: float = INFER_MIX) -> torch.Tensor:
        """[N, 33] fine SDF positions (t from each ray's origin) from 64 coarse evaluations."""
        return sample_fine(rays, interval, self.coarse_density(rays, origin, direction, interval), uniform_mix)

    def render(self, rays, origin, direction, sdf_grid, data, reso, interval, k, mode="fixed",
               transmittance="product"):
        """Colour of every ray with 64 coarse MLP points + 32 fine render samples."""
        t = self.sample(rays, origin, direction, interval)
        return fused.render_forward(rays, origin, direction, sdf_grid, data, reso, interval, k, mode, transmittance,
                                    tlist=t)

    # ---- training
    def gradients(self, points: torch.Tensor) -> float:
        """Accumulate the loss gradient over points [P,4] into self.grad; returns the loss."""
        self.loss.zero_()
        call("qsdvr_mlp_train", _p(points), points.shape[0], _p(self.params_bf16), float(self.under_weight),
             _p(self.grad), _p(self.loss), _stream(self.device))
        return self.loss

    def train_step(self, points: torch.Tensor):
        """One Adam step (fused kernel: fp32 masters, bf16 copy refreshed, grad zeroed)."""
        loss = self.gradients(points)
        self.step_count += 1
        adam_step(self.params, self.grad, self.m, self.v, self.step_count, self.lr, param_bf16=self.params_bf16)
        return loss

    def _buffer(self, name, shape, dtype):
        buf = self._bufs.get(name)
        if buf is None or buf.shape != shape:
            buf = torch.empty(shape, dtype=dtype, device=self.device)
            self._bufs[name] = buf
        return buf

    def online_step(self, rays, origin, direction, sdf_grid, data, reso, interval, k, mode="fixed",
                    transmittance="product", points: int = 65536, seed: int | None = None):
        """Online training from the renderer: a uniform-march forward over ``rays`` writes each
        render sample's alpha (ray r's samples at r * stride), ``points`` of them are drawn at
        random as (position, density) targets, and one Adam step follows.  Five launches, no
        host synchronisation."""
        n = rays.shape[0]
        stride = max_render_samples(interval)
        off = self._bufs.get(("offsets", n, stride))
        if off is None:
            off = torch.arange(0, n * stride, stride, dtype=torch.int32, device=self.device)
            self._bufs[("offsets", n, stride)] = off
        r = self._buffer("rays", (n, 4), torch.int32)
        r.copy_(rays)
        r[:, 3] = off
        alpha = self._buffer("alpha", (n * stride,), torch.float32)
        fused.render_forward(r, origin, direction, sdf_grid, data, reso, interval, k, mode, transmittance,
                             sample_alpha=alpha)
        pts = self._buffer("points", (points, 4), torch.float32)
        seed = self.step_count if seed is None else seed
        call("qsdvr_proposal_draw", _p(r), _p(origin), _p(direction), n, float(interval), _p(alpha), alpha.numel(),
             points, int(seed) & 0xFFFFFFFF, _p(pts), _stream(self.device))
        return self.train_step(pts)


def sample_fine(rays, interval, coarse, uniform_mix: float = INFER_MIX) -> torch.Tensor:
    """[N, 33] fine SDF positions from [N, 64] coarse densities (inverse-CDF sampling of the
    coarse compositing weights mixed with ``uniform_mix`` of a uniform density)."""
    if coarse.dtype != torch.float32 or coarse.shape != (rays.shape[0], N_COARSE) or not coarse.is_contiguous():
        raise ValueError("coarse must be a contiguous float32 [N, 64] tensor")
    n = rays.shape[0]
    t = torch.empty((n, N_FINE_T), dtype=torch.float32, device=rays.device)
    call("qsdvr_proposal_sample", _p(rays), n, float(interval), float(uniform_mix), _p(coarse), _p(t),
         _stream(rays.device))
    return t


def targets(rays, origin, direction, interval, alpha) -> torch.Tensor:
    """(x, y, z, density) of every render sample from a uniform-march alpha list (entries past
    the last ray's samples stay zero)."""
    pts = torch.zeros((alpha.numel(), 4), dtype=torch.float32, device=rays.device)
    call("qsdvr_proposal_targets", _p(rays), _p(origin), _p(direction), rays.shape[0], float(interval), _p(alpha),
         alpha.numel(), _p(pts), _stream(rays.device))
    return pts


def with_offsets(rays: torch.Tensor):
    """A copy of a ray batch whose render offsets index a compact per-sample list, and the
    number of render samples (a device tensor: no host synchronisation)."""
    r = rays.clone()
    nr = torch.clamp(r[:, 0] - 1, min=0)
    off = torch.cumsum(nr, 0, dtype=torch.int64) - nr
    r[:, 2] = nr
    r[:, 3] = off.to(torch.int32)
    return r, nr.sum(dtype=torch.int64)


def max_render_samples(interval: float) -> int:
    """Upper bound of render samples per ray: the box diagonal 2 sqrt(3) over the interval."""
    return int(math.ceil(2.0 * math.sqrt(3.0) / interval)) + 2


def uniform_alpha(rays, origin, direction, sdf_grid, data, reso, interval, k, mode="fixed", transmittance="product"):
    """Uniform-march forward that also writes every render sample's alpha.  Returns (colour,
    rays with compact render offsets, alpha [capacity], render-sample count on the device)."""
    r, total = with_offsets(rays)
    alpha = torch.zeros(max(rays.shape[0] * max_render_samples(interval), 1), dtype=torch.float32,
                        device=rays.device)
    color = fused.render_forward(r, origin, direction, sdf_grid, data, reso, interval, k, mode, transmittance,
                                 sample_alpha=alpha)
    return color, r, alpha, total


def uniform_tlist(rays, interval) -> torch.Tensor:
    """The method without the network: 33 evenly spaced SDF positions over each ray's
    in-box segment (same sample count as the proposal path)."""
    L = torch.clamp(rays[:, 0] - 1, min=0).float() * interval
    return (L[:, None] * torch.linspace(0.0, 1.0, N_FINE_T, device=rays.device)[None, :]).contiguous()
