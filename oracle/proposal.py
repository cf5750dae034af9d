"""ORACLE — CPU restatement of the proposal path (density-bound MLP, coarse-to-fine sampler,
training targets).  Test infrastructure only; the product never imports it.

The proposal network has no counterpart in the reference, so this file is the
specification the CUDA kernels (qsdvr_b200/csrc/proposal.cu) are checked against:

* MLP: 32-feature encoding (p, sin/cos(pi 2^l p) for l = 0..3, a constant 1 that carries
  the layer-1 bias, 4 zeros) -> 64 ReLU -> 64 ReLU -> softplus.  Parameters are the bf16
  copy the kernels read.  The kernels round the encoding and the first hidden layer to bf16
  before the tensor-core GEMMs, and in training the two back-propagated hidden gradients as
  well (db2 is summed from the rounded layer-2 gradient, as the GEMM that yields it does);
  the oracle applies the same roundings (round to nearest even) and does every other
  operation in float64.
* Loss per point: w (log1p(s) - log1p(t))^2, w = under_weight where s < t, mean over points;
  points with a negative target are ignored (they still count in the mean's denominator).
* Sampler: coarse opacity 1 - exp(-s L/64) in 64 equal bins of the in-box segment,
  compositing weights mixed with a uniform share, fine SDF positions at the CDF quantiles k/32.
* Targets: density -log(1 - alpha) / interval at each render sample of a uniform march.

Gradients of the MLP restatement are checked against torch autograd of its own forward in
the CPU tests (the roundings act as identities in the backward, as in the kernels).
"""
from __future__ import annotations

import numpy as np
import torch

N_PARAMS = 6280
OFF_W2, OFF_B2, OFF_W3, OFF_B3 = 2048, 6144, 6208, 6272


def bf16_round(x) -> np.ndarray:
    """float32 -> nearest bfloat16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(params) -> dict:
    """Split a parameter vector (any float dtype) into float64 arrays after bf16 rounding."""
    w = bf16_round(np.asarray(params, np.float32)).astype(np.float64)
    return dict(W1=w[:OFF_W2].reshape(64, 32), W2=w[OFF_W2:OFF_B2].reshape(64, 64), b2=w[OFF_B2:OFF_W3],
                w3=w[OFF_W3:OFF_B3], b3=w[OFF_B3])


def encode(points) -> np.ndarray:
    """[P,3] float32 -> [P,32] float64 encoding (already rounded to bf16)."""
    p = np.asarray(points, np.float32)[:, :3].astype(np.float64)
    f = np.zeros((p.shape[0], 32), np.float64)
    f[:, 0:3] = p
    for l in range(4):
        for c in range(3):
            ang = np.pi * (2.0 ** l) * p[:, c]
            f[:, 3 + 6 * l + 2 * c] = np.sin(ang)
            f[:, 4 + 6 * l + 2 * c] = np.cos(ang)
    f[:, 27] = 1.0
    return bf16_round(f.astype(np.float32)).astype(np.float64)


def softplus(y):
    return np.where(y > 20.0, y, np.log1p(np.exp(np.minimum(y, 20.0))))


def forward(params, points) -> dict:
    """Density bound s [P] with the intermediates the backward needs."""
    w = unpack(params)
    x = encode(points)
    d1 = x @ w["W1"].T
    h1 = bf16_round(np.maximum(d1, 0.0).astype(np.float32)).astype(np.float64)
    z2 = h1 @ w["W2"].T + w["b2"]
    h2 = np.maximum(z2, 0.0)
    y = h2 @ w["w3"] + w["b3"]
    return dict(w=w, x=x, d1=d1, h1=h1, z2=z2, h2=h2, y=y, s=softplus(y))


def density(params, points) -> np.ndarray:
    return forward(params, points)["s"]


def train_gradients(params, points, under_weight: float, round_grads: bool = True):
    """(grad [6280] float64, loss) of the mean point loss, with the kernels' bf16 roundings
    of the back-propagated hidden gradients (``round_grads=False``: the exact gradient of
    the forward, which the CPU tests compare with autograd)."""
    rnd = (lambda v: bf16_round(v.astype(np.float32)).astype(np.float64)) if round_grads else (lambda v: v)
    pts = np.asarray(points, np.float32)
    P = pts.shape[0]
    f = forward(params, pts)
    w = f["w"]
    use = pts[:, 3] >= 0.0  # a negative target marks a point to ignore
    t = np.maximum(pts[:, 3].astype(np.float64), 0.0)
    e = np.log1p(f["s"]) - np.log1p(t)
    wgt = np.where(use, np.where(e < 0.0, under_weight, 1.0), 0.0)
    loss = float((wgt * e * e).sum() / P)
    dy = 2.0 * wgt * e / (1.0 + f["s"]) / (1.0 + np.exp(-f["y"])) / P
    g = np.zeros(N_PARAMS, np.float64)
    g[OFF_B3] = dy.sum()
    g[OFF_W3:OFF_B3] = f["h2"].T @ dy
    dh2 = np.where(f["z2"] > 0.0, dy[:, None] * w["w3"][None, :], 0.0)
    dh2b = rnd(dh2)
    g[OFF_B2:OFF_W3] = dh2b.sum(0)  # db2 comes out of the bf16 dW2 GEMM (H1's constant feature)
    g[OFF_W2:OFF_B2] = (dh2b.T @ f["h1"]).reshape(-1)
    dh1 = np.where(f["d1"] > 0.0, dh2b @ w["W2"], 0.0)
    dh1b = rnd(dh1)
    g[:OFF_W2] = (dh1b.T @ f["x"]).reshape(-1)
    return g, loss


def forward_torch(params: torch.Tensor, points: torch.Tensor) -> torch.Tensor:
    """The same forward in float64 torch (roundings applied to values only), for autograd."""
    def rnd(v):
        return v + (torch.from_numpy(bf16_round(v.detach().float().numpy())).double() - v).detach()

    w = params
    x = torch.from_numpy(encode(points.numpy()))
    W1, W2 = w[:OFF_W2].reshape(64, 32), w[OFF_W2:OFF_B2].reshape(64, 64)
    h1 = rnd(torch.relu(x @ W1.T))
    h2 = torch.relu(h1 @ W2.T + w[OFF_B2:OFF_W3])
    y = h2 @ w[OFF_W3:OFF_B3] + w[OFF_B3]
    return torch.nn.functional.softplus(y, threshold=20.0)


def loss_torch(params: torch.Tensor, points: torch.Tensor, under_weight: float) -> torch.Tensor:
    s = forward_torch(params, points)
    t = torch.clamp(points[:, 3].double(), min=0.0)
    e = torch.log1p(s) - torch.log1p(t)
    wgt = torch.where(e < 0.0, torch.full_like(e, under_weight), torch.ones_like(e)) * (points[:, 3] >= 0.0).double()
    return (wgt * e * e).mean()


def coarse_points(rays, origin, direction, interval) -> np.ndarray:
    """[N*64, 3] coarse positions o + d (j + 0.5) L / 64 (float32, fused multiply-add)."""
    ns = np.asarray(rays)[:, 0].astype(np.int64)
    L = np.where(ns > 1, (ns - 1).astype(np.float32) * np.float32(interval), np.float32(0.0)).astype(np.float32)
    j = np.arange(64, dtype=np.float32)
    tt = ((j[None, :] + np.float32(0.5)) * (L[:, None] / np.float32(64.0))).astype(np.float32)
    o = np.asarray(origin, np.float32).reshape(-1, 1, 3).astype(np.float64)
    d = np.asarray(direction, np.float32).reshape(-1, 1, 3).astype(np.float64)
    p = (d * tt[..., None].astype(np.float64) + o).astype(np.float32)
    return p.reshape(-1, 3)


def sample(rays, interval, coarse_density, uniform_mix: float = 0.05) -> np.ndarray:
    """[N,33] fine SDF positions from [N,64] coarse densities (float64 restatement)."""
    ns = np.asarray(rays)[:, 0].astype(np.int64)
    L = np.where(ns > 1, (ns - 1).astype(np.float32) * np.float32(interval), np.float32(0.0)).astype(np.float64)
    dens = np.maximum(np.asarray(coarse_density, np.float64), 0.0)
    delta = L / 64.0
    keep = np.exp(-dens * delta[:, None])
    T = np.cumprod(np.concatenate([np.ones((dens.shape[0], 1)), keep[:, :-1]], 1), 1)
    wts = T * (1.0 - keep)
    tot = wts.sum(1, keepdims=True)
    pdf = np.where(tot > 0.0, (1.0 - uniform_mix) * wts / np.where(tot > 0.0, tot, 1.0) + uniform_mix / 64.0,
                   1.0 / 64.0)
    cdf = np.concatenate([np.zeros((dens.shape[0], 1)), np.cumsum(pdf, 1)], 1)
    cdf /= cdf[:, -1:]
    out = np.zeros((dens.shape[0], 33))
    q = np.arange(1, 32) / 32.0
    for r in range(dens.shape[0]):
        lo = np.clip(np.searchsorted(cdf[r], q, side="right") - 1, 0, 63)
        span = cdf[r, lo + 1] - cdf[r, lo]
        frac = np.clip(np.where(span > 0, (q - cdf[r, lo]) / np.where(span > 0, span, 1.0), 0.5), 0.0, 1.0)
        out[r, 1:32] = np.minimum((lo + frac) * delta[r], L[r])
        out[r, 32] = L[r]
    return out


def targets(rays, origin, direction, interval, alpha) -> np.ndarray:
    """[M,4] (render-sample position, -log(1 - alpha)/interval) per render sample."""
    rays = np.asarray(rays).astype(np.int64)
    o = np.asarray(origin, np.float32)
    d = np.asarray(direction, np.float32)
    # alpha clamped to [0, 1 - 1e-6] in float32, as the kernel does (the bound rounds to 0.99999899)
    a = np.clip(np.asarray(alpha, np.float32), np.float32(0.0), np.float32(1.0) - np.float32(1e-6)).astype(np.float64)
    out = np.zeros((a.shape[0], 4))
    for r in range(rays.shape[0]):
        nr, off = rays[r, 2], rays[r, 3]
        if nr <= 0:
            continue
        s = ((np.arange(nr, dtype=np.float32) + np.float32(0.5)) * np.float32(interval)).astype(np.float64)
        p = (d[r].astype(np.float64)[None, :] * s[:, None] + o[r].astype(np.float64)[None, :]).astype(np.float32)
        out[off:off + nr, :3] = p
        out[off:off + nr, 3] = -np.log1p(-a[off:off + nr]) / interval
    return out
