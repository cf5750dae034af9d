"""GPU parity of the proposal path (qsdvr_mlp_density, qsdvr_mlp_train, qsdvr_proposal_sample,
qsdvr_proposal_targets, list sampling in the fused renderer) against the CPU oracle
(oracle/proposal.py, oracle.list_points), and the gain of the trained network over the same
sample budget without it.

Tolerances: the MLP kernels and the oracle round the same values to bf16, so they differ
only where an fp32 sum lands within rounding distance of a bf16 tie: density within
1e-3 absolute + 1e-3 relative, gradients within 2e-3 norm-wise.  The sampler is float32
arithmetic against a float64 restatement: positions within 2e-4 (world units).  The list
renderer is the fused renderer: image within 1e-5, gradients within 1e-4 (as the uniform
march)."""
import numpy as np
import pytest
import torch

import oracle.oracle as O
import oracle.proposal as OP
from conftest import rel_err

pytestmark = pytest.mark.gpu
DEV = "cuda"


@pytest.fixture(scope="module")
def prop():
    from qsdvr_b200 import _lib, proposal

    _lib.lib()
    return proposal


def _params(seed=0):
    from qsdvr_b200.proposal import init_params

    w = init_params(seed, "cpu")
    g = torch.Generator().manual_seed(seed + 100)
    w[6144:6208] = (torch.rand(64, generator=g) - 0.5) * 0.2  # non-zero b2 and b3 to exercise them
    w[6272] = 0.3
    return w


def _points(n, seed=1):
    g = np.random.default_rng(seed)
    p = np.zeros((n, 4), np.float32)
    p[:, :3] = g.uniform(-1, 1, (n, 3))
    p[:, 3] = g.exponential(2.0, n) * (g.uniform(0, 1, n) < 0.5)
    p[g.uniform(0, 1, n) < 0.1, 3] = -1.0  # ignored points
    return p


def _net(prop, w):
    net = prop.ProposalNet(DEV)
    net.params.copy_(w.to(DEV))
    net.params_bf16.copy_(net.params.to(torch.bfloat16))
    return net


def _close(got, want, atol, rtol):
    got, want = np.asarray(got, np.float64), np.asarray(want, np.float64)
    return float(np.max(np.abs(got - want) / (atol + rtol * np.abs(want))))


def test_mlp_kernels_fill_the_gpu(prop):
    """The persistent MLP kernels run as many CTAs per SM as registers, shared memory and
    tensor memory allow (inference: 6 of 64 TMEM columns each, ~35 KB of shared memory and at
    most 80 registers a thread; training: 2 of 256)."""
    import ctypes

    from qsdvr_b200._lib import call

    sms = torch.cuda.get_device_properties(0).multi_processor_count
    for kernel, want in ((0, 6), (1, 2)):
        blocks, per_sm = ctypes.c_uint32(), ctypes.c_int()
        call("qsdvr_mlp_launch_shape", kernel, 1 << 24, ctypes.byref(blocks), ctypes.byref(per_sm))
        print(f"kernel {kernel}: {per_sm.value} CTAs/SM, grid {blocks.value}")
        assert per_sm.value == want and blocks.value == want * sms


@pytest.mark.parametrize("n", [1, 200, 5000])
def test_mlp_density_vs_oracle(prop, n):
    w, pts = _params(), _points(n)
    net = _net(prop, w)
    got = net.density(torch.from_numpy(pts).to(DEV)).cpu().numpy()
    want = OP.density(w.numpy(), pts)
    assert _close(got, want, 1e-3, 1e-3) <= 1.0


def test_mlp_density_ray_mode_vs_oracle(prop):
    rng = np.random.default_rng(2)
    n = 300
    rays = np.zeros((n, 4), np.int32)
    rays[:, 0] = rng.integers(0, 220, n)
    rays[:4, 0] = (0, 1, 2, 219)
    origin = rng.uniform(-0.9, 0.9, (n, 3)).astype(np.float32)
    d = rng.standard_normal((n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    w = _params(3)
    net = _net(prop, w)
    interval = 4.0 / 256
    got = net.coarse_density(*(torch.from_numpy(a).to(DEV) for a in (rays, origin, d)), interval).cpu().numpy()
    want = OP.density(w.numpy(), OP.coarse_points(rays, origin, d, interval)).reshape(n, 64)
    want[rays[:, 0] < 2] = 0.0  # rays that miss the volume
    assert _close(got, want, 1e-3, 1e-3) <= 1.0


@pytest.mark.parametrize("n", [77, 4096, 50000])  # 50000 points: 391 tiles, several per CTA
def test_mlp_train_gradients_vs_oracle(prop, n):
    w, pts = _params(4), _points(n, seed=5)
    net = _net(prop, w)
    p = torch.from_numpy(pts).to(DEV)
    net.grad.zero_()
    loss = float(net.gradients(p))
    want, want_loss = OP.train_gradients(w.numpy(), pts, net.under_weight)
    got = net.grad.cpu().numpy().astype(np.float64)
    assert abs(loss - want_loss) <= 1e-4 * max(1.0, want_loss)
    for lo, hi in ((0, 2048), (2048, 6144), (6144, 6208), (6208, 6272), (6272, 6273)):
        assert rel_err(got[lo:hi], want[lo:hi]) < 2e-3, (lo, hi)
    assert not got[6273:].any()
    # gradients accumulate into the buffer
    net.gradients(p)
    assert rel_err(net.grad.cpu().numpy(), 2 * got) < 1e-5


def test_proposal_sample_vs_oracle(prop):
    rng = np.random.default_rng(6)
    n = 500
    rays = np.zeros((n, 4), np.int32)
    rays[:, 0] = rng.integers(0, 300, n)
    rays[:3, 0] = (0, 1, 2)
    dens = rng.exponential(1.0, (n, 64)).astype(np.float32) * (rng.uniform(0, 1, (n, 64)) < 0.3)
    dens[5] = 0.0
    dens[6, 10] = 5e3
    interval = 4.0 / 256
    for mix in (0.05, 0.25, 1.0):
        got = prop.sample_fine(torch.from_numpy(rays).to(DEV), interval, torch.from_numpy(dens).to(DEV),
                               mix).cpu().numpy()
        want = OP.sample(rays, interval, dens, mix)
        assert np.abs(got - want).max() < 2e-4
        assert np.all(np.diff(got, axis=1) >= 0.0)


def test_proposal_targets_vs_oracle(prop):
    rng = np.random.default_rng(7)
    n = 64
    rays = np.zeros((n, 4), np.int32)
    rays[:, 0] = rng.integers(0, 90, n)
    nr = np.maximum(rays[:, 0] - 1, 0)
    rays[:, 2] = nr
    rays[:, 3] = np.cumsum(nr) - nr
    m = int(nr.sum())
    origin = rng.uniform(-0.9, 0.9, (n, 3)).astype(np.float32)
    d = rng.standard_normal((n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    alpha = rng.uniform(0, 1, m).astype(np.float32)
    alpha[:5] = (0.0, 1.0, 0.5, 1e-7, 0.999999)
    interval = 0.01
    got = prop.targets(*(torch.from_numpy(a).to(DEV) for a in (rays, origin, d)), interval,
                       torch.from_numpy(alpha).to(DEV)).cpu().numpy()
    want = OP.targets(rays, origin, d, interval, alpha)
    assert np.abs(got[:, :3] - want[:, :3]).max() < 1e-6
    assert _close(got[:, 3], want[:, 3], 1e-3, 1e-4) <= 1.0


def test_proposal_draw_picks_real_samples(prop):
    """Every drawn point is one of the batch's render samples with its density target; rays
    without samples are never drawn; rays are hit about uniformly."""
    from qsdvr_b200._lib import call

    rng = np.random.default_rng(8)
    n, stride = 200, 50
    rays = np.zeros((n, 4), np.int32)
    rays[:, 0] = rng.integers(0, 40, n)
    rays[:, 0][rays[:, 0] == 1] = 0
    rays[:, 2] = np.maximum(rays[:, 0] - 1, 0)
    rays[:, 3] = np.arange(n) * stride
    origin = rng.uniform(-0.9, 0.9, (n, 3)).astype(np.float32)
    d = rng.standard_normal((n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    alpha = rng.uniform(0, 0.9, n * stride).astype(np.float32)
    interval = 0.02
    dev = [torch.from_numpy(a).to(DEV) for a in (rays, origin, d, alpha)]
    count = 20000
    pts = torch.empty((count, 4), device=DEV)
    call("qsdvr_proposal_draw", dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(), n, interval,
         dev[3].data_ptr(), n * stride, count, 1234, pts.data_ptr(), None)
    from scipy.spatial import cKDTree

    got = pts.cpu().numpy().astype(np.float64)
    want = OP.targets(rays, origin, d, interval, alpha)
    rows = np.concatenate([np.arange(r * stride, r * stride + rays[r, 2]) for r in range(n)])
    dist, nearest = cKDTree(want[rows, :3]).query(got[:, :3])
    assert dist.max() < 1e-5 and (got[:, 3] >= 0.0).all()
    m = rows[nearest]
    assert np.all(np.abs(got[:, 3] - want[m, 3]) <= 1e-3 + 1e-4 * want[m, 3])
    hits = np.bincount(m // stride, minlength=n)
    has = rays[:, 2] > 0
    assert not hits[~has].any()
    expect = count / has.sum()
    assert hits[has].min() > 0.6 * expect and hits[has].max() < 1.5 * expect


def test_online_step_fits_the_renderer(prop):
    """Online training (uniform-march alphas of the batch -> drawn points -> Adam) lowers the
    loss on a scene's density."""
    from qsdvr_b200 import fused, scenes

    R, k, interval = 48, 20.0, 4.0 / 256
    grid8 = fused.pad_grid7(scenes.sphere_grid(R, 0.5, 0.0, device=DEV).reshape(-1, 7))
    data = scenes.appearance(R, seed=0, device=DEV)
    cam = _camera((3.0, 2.0, 1.5), 64, 88.9, interval, R)
    net = prop.ProposalNet(DEV, seed=1)
    losses = [float(net.online_step(cam.rayList, cam.originList, cam.dirList, grid8, data, R, interval, k,
                                    points=16384)) for _ in range(300)]
    assert np.mean(losses[-20:]) < 0.3 * np.mean(losses[:5])
    assert net.step_count == 300


def _camera(pos, size, focal, interval, R):
    from qsdvr_b200 import scenes
    from qsdvr_b200.camera import Camera

    cam = Camera(scenes.look_at(pos, size, size, focal, 2.0, 6.0), interval, R)
    cam.GenerateRayPoints(torch.ones(size * size, dtype=torch.bool))
    return cam


def _random_tlist(rays, interval, seed):
    g = np.random.default_rng(seed)
    ns = rays[:, 0].astype(np.int64)
    L = np.where(ns > 1, (ns - 1).astype(np.float32) * np.float32(interval), 0.0).astype(np.float32)
    u = np.sort(g.uniform(0, 1, (rays.shape[0], 31)), axis=1)
    t = np.concatenate([np.zeros((rays.shape[0], 1)), u, np.ones((rays.shape[0], 1))], 1) * L[:, None]
    return t.astype(np.float32)


@pytest.mark.parametrize("sh", [2, 3])
def test_list_render_vs_oracle(prop, sh):
    """Rendering at given SDF positions (33 per ray): image and gradients against the
    float64 oracle on the same sample lists."""
    from qsdvr_b200 import fused, scenes

    R, k, interval = 24, 10.0, 4.0 / 128
    cam = _camera((2.1, -3.2, 1.3), 40, 55.0, interval, R)
    grid8 = fused.pad_grid7(scenes.sphere_grid(R, 0.55, 0.01, seed=31).reshape(-1, 7)).to(DEV)
    data = scenes.appearance(R, seed=31, sh_degree=sh).to(DEV)
    rays = cam.rayList.cpu().numpy()
    tl = _random_tlist(rays, interval, 32)
    tl_d = torch.from_numpy(tl).to(DEV)
    target = torch.rand((rays.shape[0], 3), generator=torch.Generator().manual_seed(33)).to(DEV)
    sg, dg = torch.zeros_like(grid8), torch.zeros_like(data)
    img, _ = fused.render_train(target, cam.rayList, cam.originList, cam.dirList, grid8, data, R, interval, k, sg, dg,
                                mode="fixed", tlist=tl_d)
    inp = O.list_points(rays, cam.originList.cpu().numpy(), cam.dirList.cpu().numpy(), tl, R)
    inp_t = {kk: torch.from_numpy(v) for kk, v in inp.items()}
    inp_t["rayList"] = inp_t["rayList"].long()
    g7 = grid8[:, :7].double().cpu().requires_grad_()
    dd = data.double().cpu().requires_grad_()
    want = O.render(g7, dd, inp_t, k, compat=False, sh_degree=sh)
    loss = ((want - target.double().cpu()) ** 2).mean()
    wg, wd = torch.autograd.grad(loss, (g7, dd))
    assert (img.cpu().double() - want.detach()).abs().max().item() < 1e-5
    assert rel_err(sg[:, :7].cpu(), wg) < 1e-4
    assert rel_err(dg.cpu(), wd) < 1e-4
    # forward-only and backward-only kernels agree with the one-launch step
    img2 = fused.render_forward(cam.rayList, cam.originList, cam.dirList, grid8, data, R, interval, k, "fixed",
                                tlist=tl_d)
    assert (img2 - img).abs().max().item() < 1e-6
    sg2, dg2 = torch.zeros_like(grid8), torch.zeros_like(data)
    fused.render_backward((2.0 / img.numel()) * (img - target), cam.rayList, cam.originList, cam.dirList, grid8, data,
                          R, interval, k, sg2, dg2, "fixed", tlist=tl_d)
    assert rel_err(sg2.cpu(), sg.cpu()) < 1e-5 and rel_err(dg2.cpu(), dg.cpu()) < 1e-5


def test_list_ray_order(prop):
    """qsdvr_ray_order_list: a permutation of the batch listing the rays by the 15-bit Morton
    code (32^3 lattice) of the point at their median SDF position tlist[:, 16], rays without
    samples last; a list-mode training launch taken in that order gives the batch order's
    colours, loss and gradients."""
    from qsdvr_b200 import _lib, fused, scenes

    R, k, interval = 24, 10.0, 4.0 / 128
    cam = _camera((1.7, -3.3, 1.5), 40, 55.0, interval, R)
    grid8 = fused.pad_grid7(scenes.sphere_grid(R, 0.55, 0.01, seed=35).reshape(-1, 7)).to(DEV)
    data = scenes.appearance(R, seed=35).to(DEV)
    rays = cam.rayList.cpu().numpy()
    n = rays.shape[0]
    tl = _random_tlist(rays, interval, 36)
    tl_d = torch.from_numpy(tl).to(DEV)
    args = (cam.rayList, cam.originList, cam.dirList)
    order = fused.ray_order(*args, interval, tlist=tl_d)
    assert torch.equal(order.sort().values.cpu(), torch.arange(n, dtype=torch.int32))
    o, d = cam.originList.cpu().numpy(), cam.dirList.cpu().numpy()
    ns = rays[:, 0].astype(np.int64)
    pt = o + d * tl[:, 16:17]
    q = np.clip(np.floor((pt + 1.0) * 16.0), 0, 31).astype(np.int64)
    key = np.zeros(n, np.int64)
    for b in range(5):
        for a in range(3):
            key |= ((q[:, a] >> b) & 1) << (3 * b + a)
    key[ns < 2] = 1 << 15
    ks = key[order.cpu().numpy()]
    # (float rounding at lattice edges aside; rays without samples carry the largest key)
    assert np.mean(np.diff(ks) >= 0) > 0.999
    target = torch.rand((n, 3), generator=torch.Generator().manual_seed(37)).to(DEV)
    out = []
    for o_ in (None, order):
        sg, dg = torch.zeros_like(grid8), torch.zeros_like(data)
        col, loss = fused.render_train(target, *args, grid8, data, R, interval, k, sg, dg, mode="fixed",
                                       tlist=tl_d, order=o_)
        out.append((col, loss, sg, dg))
    (c0, l0, s0, d0), (c1, l1, s1, d1) = out
    assert (c0 - c1).abs().max().item() < 1e-6
    assert abs(l0.item() - l1.item()) <= n * 2.0 ** -24 * max(1.0, l0.item())
    assert rel_err(s1.cpu(), s0.cpu()) < 1e-5 and rel_err(d1.cpu(), d0.cpu()) < 1e-5
    assert _lib.device_error() == 0
    with pytest.raises(ValueError):
        fused.ray_order(*args, interval, tlist=tl_d[:, :32].contiguous())


def test_sample_alpha_matches_oracle(prop):
    from qsdvr_b200 import fused, scenes

    R, k, interval = 24, 10.0, 4.0 / 128
    cam = _camera((-2.4, 2.9, 1.1), 32, 44.0, interval, R)
    grid8 = fused.pad_grid7(scenes.sphere_grid(R, 0.5, 0.01, seed=34).reshape(-1, 7)).to(DEV)
    data = scenes.appearance(R, seed=34).to(DEV)
    color, rays, alpha, total = prop.uniform_alpha(cam.rayList, cam.originList, cam.dirList, grid8, data, R,
                                                   interval, k)
    alpha = alpha[:int(total)]
    inp = {kk: v.cpu() for kk, v in cam.GetRayPoints().items()}
    sdf = O.sample_sdf(grid8[:, :7].double().cpu(), inp["sdfPointList"], inp["sdfIndexList"], R)
    rgb = torch.zeros((inp["renderPointList"].shape[0], 3), dtype=torch.float64)
    _, want_alpha, _ = O.ray_aggregate(rgb, sdf, inp["rayList"].long(), k)
    # compact offsets (one render sample per SDF interval) match the camera's own layout
    assert torch.equal(rays[:, 3].cpu(), cam.rayList[:, 3].cpu())
    assert np.abs(alpha.cpu().numpy() - want_alpha.numpy()).max() < 1e-5


def _psnr(a, b):
    return float(-10.0 * torch.log10(((a - b) ** 2).mean().clamp_min(1e-12)))


def test_trained_proposal_beats_same_budget_without_it(prop):
    """Train the proposal MLP on the renderer's own per-sample alphas, then render a held-out
    view with 64 coarse MLP points + 32 fine samples and with 32 evenly spaced samples (the
    method without the network, same render budget).  Both are measured against the
    512-sample uniform march: the trained network must be closer to it by a wide margin."""
    from qsdvr_b200 import fused, scenes

    R, k = 64, 50.0
    interval = 4.0 / 512
    grid8 = fused.pad_grid7(scenes.procedural_grid(R, seed=0, device=DEV).reshape(-1, 7))
    data = scenes.appearance(R, seed=0, device=DEV, procedural=True)
    net = prop.ProposalNet(DEV, seed=0)
    cams = [_camera(p, 64, 88.9, interval, R)
            for p in ((4.0, 0.0, 0.5), (0.0, 4.0, 1.5), (-2.8, -2.8, 0.8), (0.5, -3.5, 2.0))]
    pool = []
    for c in cams:
        _, r, a, total = prop.uniform_alpha(c.rayList, c.originList, c.dirList, grid8, data, R, interval, k, "fixed")
        pool.append(prop.targets(r, c.originList, c.dirList, interval, a)[:int(total)])
    pool = torch.cat(pool)
    gen = torch.Generator(device=DEV).manual_seed(0)
    first = None
    for step in range(600):
        idx = torch.randint(0, pool.shape[0], (16384,), generator=gen, device=DEV)
        loss = float(net.train_step(pool[idx].contiguous()))
        first = loss if first is None else first
    assert loss < 0.25 * first
    held = _camera((2.3, 2.9, 1.9), 100, 138.9, interval, R)
    args = (held.rayList, held.originList, held.dirList)
    full = fused.render_forward(*args, grid8, data, R, interval, k, "fixed")
    t_prop = net.sample(*args, interval)
    img_prop = fused.render_forward(*args, grid8, data, R, interval, k, "fixed", tlist=t_prop)
    img_flat = fused.render_forward(*args, grid8, data, R, interval, k, "fixed",
                                    tlist=prop.uniform_tlist(held.rayList, interval))
    p_prop, p_flat = _psnr(img_prop, full), _psnr(img_flat, full)
    print(f"PSNR vs 512-sample march: proposal {p_prop:.2f} dB, uniform-32 {p_flat:.2f} dB")
    assert p_prop > p_flat + 3.0


def test_bounded_wait_gives_up_and_reports(prop):
    """The tensor-core kernels' mbarrier waits are bounded: a wait that nothing completes gives
    up after its limit (10 ms here), sets QSDVR_DEVERR_TIMEOUT and returns, and the context
    stays usable (an MLP launch right after still matches the oracle)."""
    import ctypes
    import time

    from qsdvr_b200 import _lib
    from qsdvr_b200._lib import QSDVR_DEVERR_TIMEOUT, call

    assert _lib.device_error() == 0
    done = torch.full((1,), 7, dtype=torch.int32, device=DEV)
    stream = torch.cuda.current_stream()
    t0 = time.perf_counter()
    call("qsdvr_check_bounded_wait", 10_000_000, done.data_ptr(), ctypes.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    assert int(done.item()) == 0
    assert 0.005 < elapsed < 1.0
    assert _lib.device_error() & QSDVR_DEVERR_TIMEOUT
    assert _lib.device_error() == 0  # read and cleared
    w, pts = _params(), _points(300)
    got = _net(prop, w).density(torch.from_numpy(pts).to(DEV)).cpu().numpy()
    assert _close(got, OP.density(w.numpy(), pts), 1e-3, 1e-3) <= 1.0
