"""GPU parity of the separable SDF source of the fused renderer (the reference RenderGrid's
QuadricGrid parametrisation, models/render.py:172-207, without a materialised [R^3,7] grid).

* forward: bit-identical to the fused renderer on the dense grid LayerToGridForward writes;
* layer gradients: equal to the dense path's cell gradient reduced by LayerToGridBackward up
  to summation order (1e-5 relative), and to the reference's own op chain (1e-4 relative,
  offset[3] excepted: the reference never writes it, kernel/surface.cu:255,282)."""
import numpy as np
import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def _camera(pos, size, focal, interval, R):
    from qsdvr_b200 import scenes
    from qsdvr_b200.camera import Camera

    cam = Camera(scenes.look_at(pos, size, size, focal, 2.0, 6.0), interval, R)
    cam.GenerateRayPoints(torch.ones(size * size, dtype=torch.bool))
    return cam


def _layers(R, seed):
    g = torch.Generator().manual_seed(seed)
    x, y, z = (1.0 + 0.02 * torch.randn(R, generator=g) for _ in range(3))
    c = -R
    off = torch.tensor([-2.0 * c, -2.0 * c, -2.0 * c, (3.0 * c * c) ** 0.5]) + 0.5 * torch.randn(4, generator=g)
    return [t.float().contiguous().to(DEV) for t in (x, y, z, off)]


def _dense(qs, layers, R):
    from qsdvr_b200 import fused

    grid7 = torch.empty((R, R, R, 7), device=DEV)
    qs.LayerToGridForward(grid7, *layers)
    return fused.pad_grid7(grid7.reshape(-1, 7))


@pytest.fixture(scope="module")
def qs():
    from qsdvr_b200 import _lib, qsdvr

    _lib.lib()
    return qsdvr


@pytest.mark.parametrize("mode", ["compat", "fixed"])
def test_separable_forward_bit_identical_to_dense(qs, mode):
    from qsdvr_b200 import fused, scenes

    R, k, interval = 32, 0.5, 4.0 / 96
    cam = _camera((1.2, -3.6, 1.1), 48, 66.0, interval, R)
    layers = _layers(R, 1)
    data = scenes.appearance(R, seed=2).to(DEV)
    tables = fused.separable_tables(*layers)
    args = (cam.rayList, cam.originList, cam.dirList)
    dense = fused.render_forward(*args, _dense(qs, layers, R), data, R, interval, k, mode)
    sep = fused.render_forward(*args, None, data, R, interval, k, mode, sdf_layers=tables)
    assert torch.equal(dense, sep)


@pytest.mark.parametrize("mode", ["compat", "fixed"])
def test_separable_gradients_match_dense_path(qs, mode):
    from qsdvr_b200 import fused, scenes

    R, k, interval = 32, 0.5, 4.0 / 96
    cam = _camera((-2.4, 2.9, 1.0), 48, 66.0, interval, R)
    layers = _layers(R, 3)
    data = scenes.appearance(R, seed=4).to(DEV)
    target = torch.rand((cam.rayList.shape[0], 3), generator=torch.Generator().manual_seed(5)).to(DEV)
    args = (cam.rayList, cam.originList, cam.dirList)
    grid8 = _dense(qs, layers, R)
    sg, dg = torch.zeros_like(grid8), torch.zeros_like(data)
    c0, l0 = fused.render_train(target, *args, grid8, data, R, interval, k, sg, dg, mode)
    want = [torch.empty(R, device=DEV) for _ in range(3)] + [torch.empty(4, device=DEV)]
    qs.LayerToGridBackward(sg[:, :7].contiguous().reshape(R, R, R, 7), *want)
    tables = fused.separable_tables(*layers)
    tg, dg2 = torch.zeros_like(tables), torch.zeros_like(data)
    c1, l1 = fused.render_train(target, *args, None, data, R, interval, k, tg, dg2, mode, sdf_layers=tables)
    got = fused.separable_grad(tg)
    assert torch.equal(c0, c1)
    # the same colours, their squared errors summed by float atomics in launch order: the two
    # sums differ by at most the float32 summation bound n * 2^-24 of the total
    n = cam.rayList.shape[0]
    assert abs(l0.item() - l1.item()) <= n * 2.0 ** -24 * max(1.0, l0.item())
    assert rel_err(dg2.cpu(), dg.cpu()) < 1e-6
    for g, w in zip(got, want):
        assert rel_err(g.cpu(), w.cpu()) < 1e-5


def test_separable_model_vs_reference_chain(qs):
    """SeparableRenderGrid (one fused train launch) against the reference's LayerToGrid ->
    SampleSDF / SampleNormal -> GridInterpolation -> Shader -> RayAggregate chain and its
    backward, on the same layers, appearance grid and rays."""
    from oracle.build_ref import load_reference, reference_layer_to_grid_backward
    from qsdvr_b200 import fused
    from tests.golden.make_golden import reference_render

    ref = load_reference()
    if ref is None:
        pytest.skip("reference build absent")
    R, k, interval = 32, 0.5, 4.0 / 64
    cam = _camera((1.0, -3.8, 0.9), 64, 90.0, interval, R)
    model = fused.SeparableRenderGrid(R, k, interval, mode="compat", device=DEV)
    with torch.no_grad():
        gen = torch.Generator().manual_seed(5)
        model.xLayer.add_((0.01 * torch.randn(R, generator=gen)).to(DEV))
        model.renderData.add_((0.05 * torch.randn(model.renderData.shape, generator=gen)).to(DEV))
    target = torch.rand((cam.rayList.shape[0], 3), generator=torch.Generator().manual_seed(6)).to(DEV)
    color, _ = model.train_step(target, cam.rayList, cam.originList, cam.dirList)
    # the reference chain on its own sample lists and grid
    grid = torch.empty((R, R, R, 7), device=DEV)
    ref.LayerToGridForward(grid, model.xLayer.detach().cpu().clone(), model.yLayer.detach().cpu().clone(),
                           model.zLayer.detach().cpu().clone(), model.offset.detach().cpu().clone())
    inp = cam.GetRayPoints()
    want_img, ggrid, gdata = reference_render(ref, grid.reshape(-1, 7), model.renderData.detach(), inp, R, k, target)
    assert (color - want_img).abs().max().item() < 1e-5
    assert rel_err(model.renderData.grad.cpu(), gdata.cpu()) < 1e-4
    bx, by, bz, bo = reference_layer_to_grid_backward(ref, ggrid.reshape(R, R, R, 7), R)
    assert rel_err(model.xLayer.grad.cpu(), bx) < 1e-4
    assert rel_err(model.yLayer.grad.cpu(), by) < 1e-4
    assert rel_err(model.zLayer.grad.cpu(), bz) < 1e-4
    assert rel_err(model.offset.grad[:3].cpu(), bo) < 1e-4
    # offset[3]: the sum of every cell's a6 gradient
    s6 = ggrid.reshape(-1, 7)[:, 6].sum().item()
    assert abs(model.offset.grad[3].item() - s6) < 1e-4 * max(1.0, ggrid.reshape(-1, 7)[:, 6].abs().sum().item())


def test_separable_autograd_matches_train_step(qs):
    from qsdvr_b200 import fused

    R, k, interval = 24, 2.0, 4.0 / 80
    cam = _camera((2.8, 2.2, -1.4), 40, 55.0, interval, R)
    target = torch.rand((cam.rayList.shape[0], 3), generator=torch.Generator().manual_seed(7)).to(DEV)
    a = fused.SeparableRenderGrid(R, k, interval, mode="fixed", device=DEV)
    b = fused.SeparableRenderGrid(R, k, interval, mode="fixed", device=DEV)
    img = a(cam.rayList, cam.originList, cam.dirList)
    ((img - target) ** 2).mean().backward()
    col, loss = b.train_step(target, cam.rayList, cam.originList, cam.dirList)
    assert (col - img.detach()).abs().max().item() < 1e-6
    for p, q in zip(a.parameters(), b.parameters()):
        assert rel_err(p.grad.cpu(), q.grad.cpu()) < 1e-5


def test_separable_training_driver_improves_heldout_psnr():
    """train.py --model separable: the reference's own parametrisation (layers + offset +
    appearance grid) trained through the fused kernels improves the held-out PSNR."""
    from qsdvr_b200 import train

    a = train.parser().parse_args([])
    a.model, a.reso, a.views, a.size, a.rays, a.steps = "separable", 32, 3, 48, 2048, 40
    a.interval, a.log_every = 4.0 / 96, 10 ** 9
    out = train.run(a, quiet=True)
    # measured +0.8 dB at these settings: the separable SDF (a sum of three 1-D piecewise
    # quadratics) fits the procedural scene far less than a dense grid does
    assert out["heldout_psnr_end"] > out["heldout_psnr_start"] + 0.3, out
    from qsdvr_b200 import _lib

    assert _lib.device_error() == 0
