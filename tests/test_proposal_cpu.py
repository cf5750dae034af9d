"""CPU checks of the proposal-path oracle (oracle/proposal.py): bf16 rounding, the MLP
gradient against autograd, sampler and target properties, list-sampling points."""
import numpy as np
import pytest
import torch

import oracle.oracle as O
import oracle.proposal as OP


def _params(seed=0):
    g = np.random.default_rng(seed)
    w = np.zeros(OP.N_PARAMS, np.float32)
    w[:2048] = g.uniform(-1, 1, 2048) / np.sqrt(28)
    w[2048:6144] = g.uniform(-1, 1, 4096) / 8.0
    w[6144:6208] = g.uniform(-0.1, 0.1, 64)
    w[6208:6272] = g.uniform(-1, 1, 64) / 8.0
    w[6272] = 0.3
    return w


def _points(n, seed=1):
    g = np.random.default_rng(seed)
    p = np.zeros((n, 4), np.float32)
    p[:, :3] = g.uniform(-1, 1, (n, 3))
    p[:, 3] = g.exponential(2.0, n)
    return p


def test_bf16_round_matches_torch():
    x = np.random.default_rng(0).standard_normal(10000).astype(np.float32) * 10.0 ** np.random.default_rng(1).uniform(
        -5, 5, 10000).astype(np.float32)
    want = torch.from_numpy(x).to(torch.bfloat16).float().numpy()
    assert np.array_equal(OP.bf16_round(x), want)


def test_encoding_layout():
    f = OP.encode(np.array([[0.25, -0.5, 0.0]], np.float32))[0]
    assert f[0] == 0.25 and f[1] == -0.5 and f[2] == 0.0
    assert f[27] == 1.0 and not f[28:].any()
    assert abs(f[3] - np.sin(np.pi * 0.25)) < 4e-3 and abs(f[4] - np.cos(np.pi * 0.25)) < 4e-3
    assert abs(f[3 + 6 * 3 + 2] - np.sin(8 * np.pi * -0.5)) < 4e-3


def test_mlp_gradient_matches_autograd():
    w, pts = _params(), _points(300)
    g, loss = OP.train_gradients(w, pts, 4.0, round_grads=False)
    wt = torch.from_numpy(OP.bf16_round(w).astype(np.float64)).requires_grad_()
    lt = OP.loss_torch(wt, torch.from_numpy(pts), 4.0)
    (gt,) = torch.autograd.grad(lt, wt)
    assert abs(loss - lt.item()) < 1e-12 * max(1.0, loss)
    gt = gt.numpy()
    gt[28:2048:32] = gt[29:2048:32] = gt[30:2048:32] = gt[31:2048:32] = 0.0  # zero encoding features
    assert np.abs(g[:6273] - gt[:6273]).max() / np.abs(gt).max() < 1e-10
    # the kernels' bf16 rounding of the hidden gradients moves them by less than a percent
    gr, _ = OP.train_gradients(w, pts, 4.0)
    assert np.abs(gr - g).max() / np.abs(g).max() < 1e-2


def test_sampler_properties():
    rng = np.random.default_rng(3)
    n = 64
    rays = np.zeros((n, 4), np.int32)
    rays[:, 0] = rng.integers(0, 200, n)
    rays[0, 0], rays[1, 0], rays[2, 0] = 0, 1, 150
    dens = rng.exponential(1.0, (n, 64))
    dens[3] = 0.0
    dens[2] = 0.0
    dens[2, 40] = 1e4  # an opaque bin: most fine samples land in it
    t = OP.sample(rays, 4.0 / 256, dens)
    L = np.where(rays[:, 0] > 1, (rays[:, 0] - 1) * np.float32(4.0 / 256), 0.0)
    assert np.all(np.diff(t, axis=1) >= -1e-12)
    assert np.all(t[:, 0] == 0.0) and np.allclose(t[:, 32], L)
    assert not t[0].any() and not t[1].any()
    if rays[3, 0] > 1:
        assert np.allclose(t[3], np.arange(33) * L[3] / 32)  # no density: uniform
    inside = ((t[2, 1:32] >= 40 * L[2] / 64) & (t[2, 1:32] <= 41 * L[2] / 64)).sum()
    assert inside >= 28


def test_targets_invert_alpha():
    rays = np.array([[5, 0, 4, 0], [0, 5, 0, 4], [3, 5, 2, 4]], np.int32)
    origin = np.array([[0.1, 0.2, -0.9], [0, 0, 0], [-0.5, 0.0, 0.5]], np.float32)
    direction = np.array([[0.0, 0.0, 1.0], [1, 0, 0], [0.6, 0.8, 0.0]], np.float32)
    alpha = np.array([0.0, 0.1, 0.5, 0.9, 0.2, 0.3], np.float64)
    pts = OP.targets(rays, origin, direction, 0.1, alpha)
    assert np.allclose(1.0 - np.exp(-pts[:, 3] * 0.1), alpha)
    assert np.allclose(pts[1, :3], [0.1, 0.2, -0.9 + 0.15])
    assert np.allclose(pts[5, :3], [-0.5 + 0.6 * 0.15, 0.8 * 0.15, 0.5])


def test_list_points_lie_on_the_ray():
    rng = np.random.default_rng(5)
    n = 20
    rays = np.zeros((n, 4), np.uint32)
    rays[:, 0] = rng.integers(0, 60, n)
    origin = rng.uniform(-0.5, 0.5, (n, 3)).astype(np.float32)
    d = rng.standard_normal((n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    L = np.maximum(rays[:, 0].astype(np.float32) - 1, 0) * np.float32(0.01)
    t = (L[:, None] * np.linspace(0, 1, 33)[None, :]).astype(np.float32)
    R = 16
    inp = O.list_points(rays, origin, d, t, R)
    hit = rays[:, 0] >= 2
    assert inp["sdfIndexList"].shape[0] == 33 * hit.sum() and inp["renderIndexList"].shape[0] == 32 * hit.sum()
    assert np.array_equal(inp["rayList"][:, 0], np.where(hit, 33, 0))
    # cell + local coordinate reconstruct the world point o + d t
    k = 0
    for r in np.nonzero(hit)[0]:
        idx = inp["sdfIndexList"][33 * k:33 * k + 33].astype(np.int64)
        cell = np.stack([idx % R, (idx // R) % R, idx // (R * R)], 1)
        world = (inp["sdfPointList"][33 * k:33 * k + 33] + 2 * cell + 1 - R) / R
        want = origin[r][None, :] + d[r][None, :] * t[r][:, None]
        assert np.abs(world - want).max() < 1e-5
        k += 1
