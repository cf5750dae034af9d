"""GPU parity of the fused render kernels (qsdvr_render_forward / _backward / _train).

compat mode is checked against the reference itself (golden pipeline + live build):
image within 1e-5 absolute, gradients within 1e-4 relative (max-abs error over max-abs
value).  fixed mode and BF16 storage are checked against the float64 oracle, whose
gradients are torch autograd."""
import numpy as np
import pytest
import torch

import oracle.oracle as O
from conftest import rel_err

pytestmark = pytest.mark.gpu
DEV = "cuda"
IMG_TOL = 1e-5
GRAD_TOL = 1e-4


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


@pytest.fixture(scope="module")
def fz():
    from qsdvr_b200 import _lib, fused

    _lib.lib()
    return fused


def camera_batch(pos, size, focal, interval, R, mask=None):
    """Rays of one camera through the drop-in RayCut (bit-exact with the reference)."""
    from qsdvr_b200 import scenes
    from qsdvr_b200.camera import Camera

    args = scenes.look_at(pos, size, size, focal, 2.0, 6.0)
    cam = Camera(args, interval, R)
    cam.GenerateRayPoints(torch.ones(size * size, dtype=torch.bool) if mask is None else mask)
    return cam


def oracle_inputs(cam):
    d = cam.GetRayPoints()
    inp = {k: v.cpu() for k, v in d.items() if k != "rayList"}
    inp["rayList"] = d["rayList"].cpu().long()
    return inp


def oracle_render(grid8, data, cam, R, k, compat, target=None):
    """float64 oracle image and (if target) MSE gradients w.r.t. the grids."""
    g7 = grid8[:, :7].double().cpu().requires_grad_()
    dd = data.double().cpu().requires_grad_()
    img = O.render(g7, dd, oracle_inputs(cam), k, compat)
    if target is None:
        return img.detach(), None, None
    loss = ((img - target.double().cpu()) ** 2).mean()
    gg, gd = torch.autograd.grad(loss, (g7, dd))
    return img.detach(), gg, gd


def test_fused_compat_vs_golden_pipeline(fz, golden_pipeline):
    g = golden_pipeline
    R, k, interval = g["params"]
    R = int(R)
    rays, origin, direction = _t(g["in_rays"]), _t(g["in_origin"]), _t(g["in_dir"])
    grid8 = fz.pad_grid7(_t(g["grid7"]))
    data = _t(g["data"])
    target = _t(g["target"])
    img = fz.render_forward(rays, origin, direction, grid8, data, R, interval, k)
    assert np.abs(img.cpu().numpy() - g["image"]).max() < IMG_TOL
    sg, dg = torch.zeros_like(grid8), torch.zeros_like(data)
    fz.render_backward((2.0 / img.numel()) * (img - target), rays, origin, direction, grid8, data, R, interval, k, sg,
                       dg)
    assert rel_err(sg[:, :7].cpu(), g["grid7_grad"]) < GRAD_TOL
    assert rel_err(dg.cpu(), g["data_grad"]) < GRAD_TOL
    assert float(sg[:, 7].abs().max()) == 0.0
    # the one-launch training step gives the same colour, gradients and loss
    sg2, dg2 = torch.zeros_like(grid8), torch.zeros_like(data)
    col, loss = fz.render_train(target, rays, origin, direction, grid8, data, R, interval, k, sg2, dg2)
    assert (col - img).abs().max().item() < 1e-6  # another instantiation: FMA contraction may differ
    assert rel_err(sg2.cpu(), sg.cpu()) < 1e-6 and rel_err(dg2.cpu(), dg.cpu()) < 1e-6
    assert abs(loss.item() - ((img - target) ** 2).sum().item()) < 1e-4 * max(1.0, loss.item())


def test_fused_compat_vs_reference_live(fz):
    from oracle.build_ref import load_reference
    from qsdvr_b200 import scenes
    from tests.golden.make_golden import reference_render

    ref = load_reference()
    if ref is None:
        pytest.skip("reference build absent")
    R, k, interval = 64, 10.0, 4.0 / 256  # up to ~220 samples per ray: 7 chunks
    cam = camera_batch((0.3, -4.0, 0.4), 100, 138.9, interval, R)
    inp = cam.GetRayPoints()
    grid7 = scenes.sphere_grid(R, 0.5, 0.01, seed=1).reshape(-1, 7).to(DEV)
    data = scenes.appearance(R, seed=1).to(DEV)
    target = torch.rand((cam.rayList.shape[0], 3), generator=torch.Generator().manual_seed(2)).to(DEV)
    want_img, want_g7, want_data = reference_render(ref, grid7, data, inp, R, k, target)
    grid8 = fz.pad_grid7(grid7)
    sg, dg = torch.zeros_like(grid8), torch.zeros_like(data)
    img, _ = fz.render_train(target, cam.rayList, cam.originList, cam.dirList, grid8, data, R, interval, k, sg, dg)
    e_img = (img - want_img).abs().max().item()
    e_g, e_d = rel_err(sg[:, :7].cpu(), want_g7.cpu()), rel_err(dg.cpu(), want_data.cpu())
    print(f"\ncompat vs the reference build (R={R}, {cam.rayList.shape[0]} rays): image {e_img:.2e}, "
          f"SDF grad {e_g:.2e}, appearance grad {e_d:.2e}")
    assert e_img < IMG_TOL
    assert e_g < GRAD_TOL
    assert e_d < GRAD_TOL


@pytest.mark.parametrize("interval", [4.0 / 64, 4.0 / 192])
def test_fused_fixed_vs_oracle(fz, interval):
    from qsdvr_b200 import scenes

    R, k = 24, 8.0
    cam = camera_batch((2.2, -3.0, 1.5), 40, 55.0, interval, R)
    grid8 = fz.pad_grid7(scenes.sphere_grid(R, 0.55, 0.01, seed=3).reshape(-1, 7)).to(DEV)
    data = scenes.appearance(R, seed=3).to(DEV)
    target = torch.rand((cam.rayList.shape[0], 3), generator=torch.Generator().manual_seed(4)).to(DEV)
    sg, dg = torch.zeros_like(grid8), torch.zeros_like(data)
    img, _ = fz.render_train(target, cam.rayList, cam.originList, cam.dirList, grid8, data, R, interval, k, sg, dg,
                             mode="fixed")
    want, wg, wd = oracle_render(grid8, data, cam, R, k, compat=False, target=target)
    e_img = (img.cpu().double() - want).abs().max().item()
    e_g, e_d = rel_err(sg[:, :7].cpu(), wg), rel_err(dg.cpu(), wd)
    print(f"\nfixed vs the float64 oracle (R={R}, interval {interval:.4f}): image {e_img:.2e}, SDF grad {e_g:.2e}, "
          f"appearance grad {e_d:.2e}")
    assert e_img < IMG_TOL
    assert e_g < GRAD_TOL
    assert e_d < GRAD_TOL


def test_fused_bf16_storage_vs_oracle(fz):
    """BF16 grids, FP32 arithmetic, compensated log-transmittance: compared with the
    float64 oracle evaluated on the same bf16-rounded grids."""
    from qsdvr_b200 import scenes

    R, k, interval = 32, 10.0, 4.0 / 128
    cam = camera_batch((-2.5, -2.9, 1.2), 48, 66.0, interval, R)
    grid8 = fz.pad_grid7(scenes.sphere_grid(R, 0.5, 0.01, seed=5).reshape(-1, 7)).to(DEV)
    data = scenes.appearance(R, seed=5).to(DEV)
    g16, d16 = fz.sdf_cells_bf16(grid8), data.to(torch.bfloat16)
    g_read = O.sdf_cells_decode(g16)  # the coefficients the kernels read from the bf16 cells
    target = torch.rand((cam.rayList.shape[0], 3), generator=torch.Generator().manual_seed(6)).to(DEV)
    for mode in ("compat", "fixed"):
        sg, dg = torch.zeros_like(grid8), torch.zeros_like(data)
        img, _ = fz.render_train(target, cam.rayList, cam.originList, cam.dirList, g16, d16, R, interval, k, sg, dg,
                                 mode=mode, transmittance="log")
        want, wg, wd = oracle_render(g_read, d16.float(), cam, R, k, compat=(mode == "compat"), target=target)
        assert (img.cpu().double() - want).abs().max().item() < IMG_TOL
        assert rel_err(sg[:, :7].cpu(), wg) < GRAD_TOL
        assert rel_err(dg.cpu(), wd) < GRAD_TOL


def test_log_transmittance_matches_product(fz):
    from qsdvr_b200 import scenes

    R, k, interval = 48, 20.0, 4.0 / 256
    cam = camera_batch((0.1, 3.9, -0.8), 64, 90.0, interval, R)
    grid8 = fz.pad_grid7(scenes.sphere_grid(R, 0.6, 0.01, seed=7).reshape(-1, 7)).to(DEV)
    data = scenes.appearance(R, seed=7).to(DEV)
    a = fz.render_forward(cam.rayList, cam.originList, cam.dirList, grid8, data, R, interval, k, "fixed", "product")
    b = fz.render_forward(cam.rayList, cam.originList, cam.dirList, grid8, data, R, interval, k, "fixed", "log")
    assert (a - b).abs().max().item() < IMG_TOL


def test_autograd_function_matches_train_kernel(fz):
    from qsdvr_b200 import scenes

    R, k, interval = 32, 6.0, 4.0 / 96
    cam = camera_batch((1.5, -3.4, 1.0), 50, 70.0, interval, R)
    model = fz.DenseRenderGrid(R, k, interval, mode="fixed", sdf_grid=scenes.sphere_grid(R, 0.5, 0.01, device=DEV),
                               data=scenes.appearance(R, device=DEV))
    target = torch.rand((cam.rayList.shape[0], 3), generator=torch.Generator().manual_seed(8)).to(DEV)
    img = model(cam.rayList, cam.originList, cam.dirList)
    loss = ((img - target) ** 2).mean()
    loss.backward()
    sg, dg = torch.zeros_like(model.sdfGrid), torch.zeros_like(model.renderData)
    col, ls = fz.render_train(target, cam.rayList, cam.originList, cam.dirList, model.sdfGrid.detach(),
                              model.renderData.detach(), R, interval, k, sg, dg, mode="fixed")
    assert (col - img.detach()).abs().max().item() < 1e-6
    # the kernel's loss is summed by float atomics in launch order: within n * 2^-24 of the total
    assert abs(ls.item() / (3 * col.shape[0]) - loss.item()) <= col.shape[0] * 2.0 ** -24 * max(1e-6, loss.item())
    assert rel_err(model.sdfGrid.grad.cpu(), sg.cpu()) < 1e-6
    assert rel_err(model.renderData.grad.cpu(), dg.cpu()) < 1e-6


def test_rays_outside_grid_are_flagged_not_faulting(fz):
    from qsdvr_b200 import _lib

    R = 8
    _lib.device_error()
    rays = torch.tensor([[10, 0, 9, 0], [0, 10, 0, 9], [5, 10, 4, 9]], dtype=torch.int32, device=DEV)
    origin = torch.tensor([[0.0, 0.0, 0.0], [0.0, 0.0, 0.0], [3.0, 0.0, 0.0]], device=DEV)  # third starts outside
    direction = torch.tensor([[1.0, 0.0, 0.0], [1.0, 0.0, 0.0], [1.0, 0.0, 0.0]], device=DEV)
    grid8 = torch.zeros((R ** 3, 8), device=DEV)
    grid8[:, 3] = 1.0
    data = torch.ones(((R + 1) ** 3, 32), device=DEV)
    img = fz.render_forward(rays, origin, direction, grid8, data, R, 0.05, 5.0)
    assert torch.isfinite(img).all()
    assert img[2].abs().max().item() == 0.0
    assert _lib.device_error() & _lib.DEVERR_INDEX


@pytest.mark.parametrize("mode", ["compat", "fixed"])
def test_persistent_stash_path_matches_one_ray_per_block(fz, mode):
    """The persistent grid (dynamic ray scheduling, per-warp row stash reloaded in the
    backward) gives the same colours, loss and gradients as one ray per block."""
    from qsdvr_b200 import scenes

    R, k, interval = 40, 12.0, 4.0 / 320  # rays up to ~250 samples: 8 chunks, beyond the stash
    cam = camera_batch((2.0, 3.1, -1.7), 72, 100.0, interval, R)
    grid8 = fz.pad_grid7(scenes.sphere_grid(R, 0.55, 0.01, seed=9).reshape(-1, 7)).to(DEV)
    data = scenes.appearance(R, seed=9).to(DEV)
    target = torch.rand((cam.rayList.shape[0], 3), generator=torch.Generator().manual_seed(9)).to(DEV)
    out = []
    for persistent in (False, True):
        sg, dg = torch.zeros_like(grid8), torch.zeros_like(data)
        col, loss = fz.render_train(target, cam.rayList, cam.originList, cam.dirList, grid8, data, R, interval, k, sg,
                                    dg, mode=mode, persistent=persistent)
        out.append((col, loss, sg, dg))
    (c0, l0, s0, d0), (c1, l1, s1, d1) = out
    assert (c0 - c1).abs().max().item() < 1e-6
    # losses summed by float atomics in launch order: within n * 2^-24 of the total
    assert abs(l0.item() - l1.item()) <= c0.shape[0] * 2.0 ** -24 * max(1.0, l0.item())
    assert rel_err(s1.cpu(), s0.cpu()) < 1e-5 and rel_err(d1.cpu(), d0.cpu()) < 1e-5


@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_fused_sh_degree3_vs_oracle(fz, storage):
    """SH degree 3 (64-channel rows, fixed mode): forward and gradients against the float64
    oracle with autograd."""
    from qsdvr_b200 import scenes

    R, k, interval = 24, 8.0, 4.0 / 160
    cam = camera_batch((-1.9, 3.2, 1.4), 40, 55.0, interval, R)
    grid8 = fz.pad_grid7(scenes.sphere_grid(R, 0.55, 0.01, seed=21).reshape(-1, 7)).to(DEV)
    data = scenes.appearance(R, seed=21, sh_degree=3).to(DEV)
    if storage == "bf16":
        gk, dk = fz.sdf_cells_bf16(grid8), data.to(torch.bfloat16)
        grid8 = torch.nn.functional.pad(O.sdf_cells_decode(gk), (0, 1)).to(DEV)
        data = dk.float()
    else:
        gk, dk = grid8, data
    target = torch.rand((cam.rayList.shape[0], 3), generator=torch.Generator().manual_seed(22)).to(DEV)
    sg, dg = torch.zeros_like(grid8), torch.zeros_like(data)
    img, _ = fz.render_train(target, cam.rayList, cam.originList, cam.dirList, gk, dk, R, interval, k, sg, dg,
                             mode="fixed", transmittance="log" if storage == "bf16" else "product")
    g7 = grid8[:, :7].double().cpu().requires_grad_()
    dd = data.double().cpu().requires_grad_()
    want = O.render(g7, dd, oracle_inputs(cam), k, compat=False, sh_degree=3)
    loss = ((want - target.double().cpu()) ** 2).mean()
    wg, wd = torch.autograd.grad(loss, (g7, dd))
    assert (img.cpu().double() - want.detach()).abs().max().item() < IMG_TOL
    assert rel_err(sg[:, :7].cpu(), wg) < GRAD_TOL
    assert rel_err(dg.cpu(), wd) < GRAD_TOL
    assert float(dg[:, 53:].abs().max()) == 0.0  # unused channels get no gradient


def test_ray_order_gives_same_results(fz):
    """Rays taken in Morton order of their midpoints (qsdvr_ray_order, args.order) give the
    same colours, loss and gradients as the batch order.  The order is a permutation that lists
    the rays by the 15-bit Morton code of their midpoint (32^3 lattice; rays without samples
    last); qsdvr_ray_order_keys gives the 30-bit codes (1024^3 lattice).  An order entry outside
    the batch is skipped and flagged, not read."""
    import numpy as np

    from qsdvr_b200 import _lib, scenes

    R, k, interval = 32, 8.0, 4.0 / 96
    cam = camera_batch((1.9, -3.1, 1.4), 56, 75.0, interval, R)
    grid8 = fz.pad_grid7(scenes.sphere_grid(R, 0.55, 0.01, seed=11).reshape(-1, 7)).to(DEV)
    data = scenes.appearance(R, seed=11).to(DEV)
    n = cam.rayList.shape[0]
    target = torch.rand((n, 3), generator=torch.Generator().manual_seed(12)).to(DEV)
    args = (cam.rayList, cam.originList, cam.dirList)
    order = fz.ray_order(*args, interval)
    assert torch.equal(order.sort().values.cpu(), torch.arange(n, dtype=torch.int32))
    r, o, d = (t.cpu().numpy() for t in args)
    ns = r[:, 0].astype(np.int64)
    t = 0.5 * (ns - 1).astype(np.float32) * np.float32(interval)
    mid = o + d * t[:, None]

    def morton(bits, none):
        q = np.clip(np.floor((mid + 1.0) * (1 << (bits - 1))), 0, (1 << bits) - 1).astype(np.int64)
        key = np.zeros(n, np.int64)
        for b in range(bits):
            for a in range(3):
                key |= ((q[:, a] >> b) & 1) << (3 * b + a)
        key[ns < 2] = none
        return key

    # the order: 15-bit codes non-decreasing (float rounding at lattice edges aside)
    ks = morton(5, 1 << 15)[order.cpu().numpy()]
    assert np.all(np.diff(ks) >= 0) or np.mean(np.diff(ks) >= 0) > 0.999
    # the keys entry point: 30-bit codes
    k30 = fz.ray_order_keys(*args, interval).cpu().numpy().astype(np.int64)
    assert np.mean(k30 == morton(10, 0x7FFFFFFF)) > 0.999
    out = []
    for o_ in (None, order):
        sg, dg = torch.zeros_like(grid8), torch.zeros_like(data)
        col, loss = fz.render_train(target, *args, grid8, data, R, interval, k, sg, dg, mode="fixed", order=o_)
        out.append((col, loss, sg, dg))
    (c0, l0, s0, d0), (c1, l1, s1, d1) = out
    assert (c0 - c1).abs().max().item() < 1e-6
    assert abs(l0.item() - l1.item()) <= n * 2.0 ** -24 * max(1.0, l0.item())
    assert rel_err(s1.cpu(), s0.cpu()) < 1e-5 and rel_err(d1.cpu(), d0.cpu()) < 1e-5
    assert _lib.device_error() == 0
    bad = order.clone()
    bad[0] = n + 5
    fz.render_forward(*args, grid8, data, R, interval, k, "fixed", order=bad)
    assert _lib.device_error() & _lib.QSDVR_DEVERR_RAY


def test_bf16_data_gradient(fz):
    """data_grad_storage bf16: the same colours and SDF gradient as with an fp32 data
    gradient, and the appearance gradient within the rounding of bf16 accumulation (each
    vertex row receives a few contributions per batch: 2e-2 relative)."""
    from qsdvr_b200 import _lib, scenes

    R, k, interval = 32, 8.0, 4.0 / 96
    cam = camera_batch((-2.0, 3.0, 1.6), 56, 75.0, interval, R)
    grid8 = fz.pad_grid7(scenes.sphere_grid(R, 0.55, 0.01, seed=13).reshape(-1, 7)).to(DEV)
    data = scenes.appearance(R, seed=13).to(DEV)
    target = torch.rand((cam.rayList.shape[0], 3), generator=torch.Generator().manual_seed(14)).to(DEV)
    args = (cam.rayList, cam.originList, cam.dirList)
    res = []
    for dt in (torch.float32, torch.bfloat16):
        for storage in ("f32", "bf16"):
            g = (grid8, data) if storage == "f32" else (fz.sdf_cells_bf16(grid8), data.to(torch.bfloat16))
            sg, dg = torch.zeros_like(grid8), torch.zeros(data.shape, dtype=dt, device=DEV)
            col, _ = fz.render_train(target, *args, *g, R, interval, k, sg, dg, mode="fixed",
                                     transmittance="product" if storage == "f32" else "log")
            res.append((storage, dt, col, sg, dg))
    by = {(s, d): (c, sg, dg) for s, d, c, sg, dg in res}
    for storage in ("f32", "bf16"):
        c32, s32, d32 = by[(storage, torch.float32)]
        c16, s16, d16 = by[(storage, torch.bfloat16)]
        assert torch.equal(c32, c16)
        assert rel_err(s16.cpu(), s32.cpu()) < 1e-5
        err = rel_err(d16.float().cpu(), d32.cpu())
        assert 0 < err < 2e-2, (storage, err)
    assert _lib.device_error() == 0


def test_edge_batches(fz):
    """Edge cases of a batch.

    * An empty batch launches nothing: empty colours, zero loss, gradients untouched.
    * Rays whose record holds 0 or 1 SDF samples render black and add no gradient.
    * A ray longer than the 8192 render samples (256 warp chunks) the fused kernels take is
      skipped before any access and flagged (QSDVR_DEVERR_RAY), rendering black.
    The other rays of the batch render and train exactly as in a batch without those three."""
    from qsdvr_b200 import _lib, scenes

    R, k, interval = 32, 8.0, 4.0 / 96
    cam = camera_batch((1.7, -3.2, 1.3), 48, 65.0, interval, R)
    grid8 = fz.pad_grid7(scenes.sphere_grid(R, 0.55, 0.01, seed=15).reshape(-1, 7)).to(DEV)
    data = scenes.appearance(R, seed=15).to(DEV)
    rays, origin, direction = cam.rayList.contiguous(), cam.originList, cam.dirList
    n = rays.shape[0]
    target = torch.rand((n, 3), generator=torch.Generator().manual_seed(16)).to(DEV)
    _lib.device_error()

    # empty batch
    e4, e3 = rays[:0].contiguous(), origin[:0].contiguous()
    assert fz.render_forward(e4, e3, e3, grid8, data, R, interval, k, "fixed").shape == (0, 3)
    sg, dg = torch.zeros_like(grid8), torch.zeros_like(data)
    col, loss = fz.render_train(target[:0], e4, e3, e3, grid8, data, R, interval, k, sg, dg, mode="fixed")
    assert col.shape == (0, 3) and float(loss) == 0.0 and not sg.any() and not dg.any()

    # three rays with samples become: no samples, one sample, too many samples
    with_samples = torch.nonzero(rays[:, 0] >= 2).reshape(-1).cpu()
    odd = with_samples[torch.tensor([0, len(with_samples) // 2, len(with_samples) - 1])]
    keep = torch.ones(n, dtype=torch.bool)
    keep[odd] = False
    mod = rays.clone()
    mod[odd, 0] = torch.tensor([0, 1, 9000], dtype=torch.int32, device=DEV)

    def train(r, o, d, t):
        sg, dg = torch.zeros_like(grid8), torch.zeros_like(data)
        col, loss = fz.render_train(t, r, o, d, grid8, data, R, interval, k, sg, dg, mode="fixed")
        return col, float(loss), sg, dg

    kd = keep.to(DEV)
    c0, l0, s0, d0 = train(rays[kd].contiguous(), origin[kd].contiguous(), direction[kd].contiguous(),
                           target[kd].contiguous())
    assert _lib.device_error() == 0
    c1, l1, s1, d1 = train(mod, origin, direction, target)
    err = _lib.device_error()
    assert err & _lib.QSDVR_DEVERR_RAY and not err & _lib.QSDVR_DEVERR_INDEX
    assert float(c1[odd.to(DEV)].abs().max()) == 0.0
    assert (c1[kd] - c0).abs().max().item() < 1e-6
    extra = float((target[odd.to(DEV)] ** 2).sum())  # the black rays' squared error
    assert abs(l1 - (l0 + extra)) <= n * 2.0 ** -24 * max(1.0, l1)
    # the gradient scale is 2 / (3 N): the same rays' gradients with N = n and N = n - 3
    scale = (n - 3) / n
    assert rel_err(s1.cpu(), (s0 * scale).cpu()) < 1e-5 and rel_err(d1.cpu(), (d0 * scale).cpu()) < 1e-5


def test_nonfinite_colour_propagates_like_the_reference(fz):
    """compat mode with non-finite values, against the reference build run live.  A cell
    whose quadric is constant (only a6 != 0) has an infinite SDF and a 0/0 normal.  alpha is
    0 across such cells, and the reference shades their samples anyway, so the rays crossing
    them get a NaN colour, and the NaN colour gradient reaches every sample of those rays.
    The fused kernel skips samples with alpha = 0, unless their normal or rgb gradient is not
    finite.  So it must give the same NaN rays and the same non-finite gradient entries, and
    the finite entries within the usual tolerances."""
    from oracle.build_ref import load_reference
    from qsdvr_b200 import scenes
    from tests.golden.make_golden import reference_render

    ref = load_reference()
    if ref is None:
        pytest.skip("reference build absent")
    R, k, interval = 16, 5.0, 4.0 / 64
    cam = camera_batch((0.3, -4.0, 0.4), 40, 55.0, interval, R)
    inp = cam.GetRayPoints()
    g = scenes.sphere_grid(R, 0.5, 0.01, seed=3).reshape(R, R, R, 7).to(DEV)  # [z][y][x]
    g[4:6] = 0.0
    g[4:6, :, :, 6] = 0.3  # a slab of constant cells, z in [-0.5, -0.25)
    grid7 = g.reshape(-1, 7).contiguous()
    data = scenes.appearance(R, seed=3).to(DEV)
    target = torch.rand((cam.rayList.shape[0], 3), generator=torch.Generator().manual_seed(4)).to(DEV)
    want_img, want_g7, want_data = reference_render(ref, grid7, data, inp, R, k, target)
    nan_rays = ~torch.isfinite(want_img).all(dim=1)
    assert nan_rays.any() and (~nan_rays).any()  # the case is exercised
    grid8 = fz.pad_grid7(grid7)
    sg, dg = torch.zeros_like(grid8), torch.zeros_like(data)
    img, _ = fz.render_train(target, cam.rayList, cam.originList, cam.dirList, grid8, data, R, interval, k, sg, dg)
    assert torch.equal(torch.isfinite(img), torch.isfinite(want_img))
    fin = torch.isfinite(want_img)
    assert (img[fin] - want_img[fin]).abs().max().item() < IMG_TOL
    assert rel_err(sg[:, :7].cpu(), want_g7.cpu()) < GRAD_TOL  # rel_err also requires equal non-finite masks
    assert rel_err(dg.cpu(), want_data.cpu()) < GRAD_TOL


@pytest.mark.parametrize("mode", ["compat", "fixed"])
def test_same_cell_merged_scatter(fz, mode):
    """merge_scatter: samples of a chunk in the same cell send one summed RED per corner row.
    With 4 samples per cell (R=32, interval 4/256) most chunks merge; colours and loss are
    untouched, both gradients equal the unmerged scatter's within float reassociation (1e-6
    norm-wise), and the bf16-accumulated gradient stays within its 2e-2."""
    from qsdvr_b200 import _lib, scenes

    R, k, interval = 32, 8.0, 4.0 / 256
    cam = camera_batch((2.3, -2.9, 1.5), 48, 66.0, interval, R)
    grid8 = fz.pad_grid7(scenes.sphere_grid(R, 0.55, 0.01, seed=31).reshape(-1, 7)).to(DEV)
    data = scenes.appearance(R, seed=31).to(DEV)
    target = torch.rand((cam.rayList.shape[0], 3), generator=torch.Generator().manual_seed(32)).to(DEV)
    args = (cam.rayList, cam.originList, cam.dirList)
    order = fz.ray_order(*args, interval)
    res = {}
    for merge in (False, True):
        for dt in (torch.float32, torch.bfloat16):
            sg, dg = torch.zeros_like(grid8), torch.zeros(data.shape, dtype=dt, device=DEV)
            col, loss = fz.render_train(target, *args, grid8, data, R, interval, k, sg, dg, mode=mode, order=order,
                                        merge=merge)
            res[(merge, dt)] = (col, loss, sg, dg)
    c0, l0, s0, d0 = res[(False, torch.float32)]
    c1, l1, s1, d1 = res[(True, torch.float32)]
    assert torch.equal(c0, c1)
    assert abs(l0.item() - l1.item()) <= c0.shape[0] * 2.0 ** -24 * max(1.0, l0.item())
    assert rel_err(s1.cpu(), s0.cpu()) < 1e-6
    e = rel_err(d1.cpu(), d0.cpu())
    assert e < 1e-6, e
    eb = rel_err(res[(True, torch.bfloat16)][3].float().cpu(), d0.cpu())
    assert eb < 2e-2, eb
    assert _lib.device_error() == 0


def test_nonfinite_appearance_row_of_inactive_samples(fz):
    """A documented divergence from the reference: a non-finite appearance row that only
    samples with alpha = 0 read.  The reference shades every sample, so NaN x 0 makes the
    colour of each ray that reads such a row NaN; the fused kernel neither gathers nor shades
    those samples, so their rows never reach a colour or a gradient.  Here every row that some
    alpha = 0 sample reads and no alpha > 0 sample reads holds NaN (compat mode, the
    reference's addressing): the kernel's colours equal those of the same model with those rows
    zeroed, bit for bit, its gradients up to the order of their float atomics, and all are
    finite; the reference (run live when built)
    gives NaN colours on the rays that read them."""
    from oracle.build_ref import load_reference
    from qsdvr_b200 import scenes
    from tests.golden.make_golden import reference_render

    R, k, interval = 16, 5.0, 4.0 / 64
    cam = camera_batch((0.3, -4.0, 0.4), 40, 55.0, interval, R)
    grid7 = scenes.sphere_grid(R, 0.5, 0.01, seed=6).reshape(-1, 7).to(DEV)
    grid8 = fz.pad_grid7(grid7)
    data = scenes.appearance(R, seed=6).to(DEV)
    pts = cam.GetRayPoints()
    alpha = torch.zeros(pts["renderIndexList"].shape[0], device=DEV)
    fz.render_forward(cam.rayList, cam.originList, cam.dirList, grid8, data, R, interval, k, "compat",
                      sample_alpha=alpha)
    R1 = R + 1
    corners = torch.tensor([0, 1, R1, R1 + 1, R1 * R1, R1 * R1 + 1, R1 * R1 + R1, R1 * R1 + R1 + 1], device=DEV)
    rows = pts["renderIndexList"].long()[:, None] + corners[None, :]  # compat: the cell index as base vertex
    rc = rows.cpu()
    assert int(rc.min()) >= 0 and int(rc.max()) < R1 ** 3  # checked on the host before indexing with them
    read_active = torch.zeros(R1 ** 3, dtype=torch.bool, device=DEV)
    read_inactive = torch.zeros_like(read_active)
    read_active[rows[alpha > 0].reshape(-1)] = True
    read_inactive[rows[alpha == 0].reshape(-1)] = True
    only_inactive = read_inactive & ~read_active
    assert int(only_inactive.sum()) > 100  # the case is exercised
    bad, zeroed = data.clone(), data.clone()
    bad[only_inactive] = float("nan")
    zeroed[only_inactive] = 0.0
    target = torch.rand((cam.rayList.shape[0], 3), generator=torch.Generator().manual_seed(7)).to(DEV)
    out = []
    for d in (bad, zeroed):
        sg, dg = torch.zeros_like(grid8), torch.zeros_like(data)
        img, loss = fz.render_train(target, cam.rayList, cam.originList, cam.dirList, grid8, d, R, interval, k, sg, dg)
        out.append((img, loss, sg, dg))
    (i0, l0, s0, d0), (i1, l1, s1, d1) = out
    assert torch.isfinite(i0).all() and torch.isfinite(s0).all() and torch.isfinite(d0).all()
    # colours bit for bit; gradients up to the order of their float atomics
    assert torch.equal(i0, i1) and rel_err(s0.cpu(), s1.cpu()) < 1e-6 and rel_err(d0.cpu(), d1.cpu()) < 1e-6
    ref = load_reference()
    if ref is not None:
        want, _, _ = reference_render(ref, grid7, bad, pts, R, k, target)
        assert (~torch.isfinite(want)).any()  # the reference's colours on those rays are NaN


@pytest.mark.parametrize("storage,sh", [("f32", 2), ("bf16", 3)])
def test_brick_staged_frame_forward(fz, storage, sh):
    """qsdvr_render_forward_bricks (TMA-staged appearance bricks, one thread per ray, rays in
    8 x 8 tiles) gives the fused forward's colours (fixed mode, log transmittance) within 1e-5,
    for rays in tile order and in pixel order (fewer rays per brick, same result)."""
    from qsdvr_b200 import _lib, scenes
    from qsdvr_b200.camera import Camera

    R, k, interval = 24, 8.0, 4.0 / 160
    grid8 = fz.pad_grid7(scenes.sphere_grid(R, 0.55, 0.01, seed=41).reshape(-1, 7)).to(DEV)
    data = scenes.appearance(R, seed=41, sh_degree=sh).to(DEV)
    if storage == "bf16":
        grid8, data = fz.sdf_cells_bf16(grid8), data.to(torch.bfloat16)
    args = scenes.look_at((-1.7, 3.1, 1.9), 64, 48, 60.0, 2.0, 6.0)
    _lib.device_error()
    for order in ("tiles", "pixels"):
        cam = Camera(args, interval, R)
        cam.GenerateRayPoints(torch.ones(64 * 48, dtype=torch.bool), order=order)
        want = fz.render_forward(cam.rayList, cam.originList, cam.dirList, grid8, data, R, interval, k, "fixed", "log")
        got = fz.render_forward_bricks(cam.rayList, cam.originList, cam.dirList, grid8, data, R, interval, k)
        assert (got - want).abs().max().item() < 1e-5, order
        assert float(want.abs().max()) > 0.05  # the frame is not empty
    assert _lib.device_error() == 0


def test_long_rays(fz):
    """Rays of ~3000 render samples (interval 2 sqrt(3) / 3500 through a 16^3 grid: ~94 warp
    chunks, beyond the 64 chunks of the earlier limit) train like the float64 oracle: image
    within 1e-5 and appearance gradient within 1e-4 relative; the persistent kernel's stash
    then covers only the last 6 chunks, and the rest are gathered again in the backward.  At
    such a small interval a sample's SDF gradient is the difference of two nearly equal terms
    (its own interval's dalpha/dsdf and the next one's), which float32 cannot resolve on every
    entry: the SDF-gradient bar of 1e-4 applies where the same formulas in float32 torch agree
    with float64 within 1e-4 of the largest entry, and at most 1 % of the entries are left out."""
    import math

    from qsdvr_b200 import _lib, scenes

    R, k, interval = 16, 6.0, 2.0 * math.sqrt(3.0) / 3500
    cam = camera_batch((2.6, -2.2, 1.9), 8, 9.0, interval, R)
    assert int(cam.rayList[:, 0].max()) > 2048
    grid8 = fz.pad_grid7(scenes.sphere_grid(R, 0.5, 0.01, seed=17).reshape(-1, 7)).to(DEV)
    data = scenes.appearance(R, seed=17).to(DEV)
    target = torch.rand((cam.rayList.shape[0], 3), generator=torch.Generator().manual_seed(18)).to(DEV)
    _lib.device_error()
    sg, dg = torch.zeros_like(grid8), torch.zeros_like(data)
    img, _ = fz.render_train(target, cam.rayList, cam.originList, cam.dirList, grid8, data, R, interval, k, sg, dg,
                             mode="fixed")
    assert _lib.device_error() == 0
    want, wg, wd = oracle_render(grid8, data, cam, R, k, compat=False, target=target)
    saved = O.DTYPE
    O.DTYPE = torch.float32
    try:
        g32 = grid8[:, :7].float().cpu().requires_grad_()
        d32 = data.float().cpu().requires_grad_()
        img32 = O.render(g32, d32, oracle_inputs(cam), k, False)
        wg32, _ = torch.autograd.grad(((img32 - target.cpu()) ** 2).mean(), (g32, d32))
    finally:
        O.DTYPE = saved
    ok = (wg32.double() - wg).abs() <= 1e-4 * wg.abs().max()
    assert (img.cpu().double() - want).abs().max().item() < IMG_TOL
    assert rel_err(dg.cpu(), wd) < GRAD_TOL
    assert int((~ok).sum()) <= 0.01 * ok.numel()
    got = sg[:, :7].cpu().double()
    assert float((got - wg)[ok].abs().max() / wg.abs().max()) < GRAD_TOL
