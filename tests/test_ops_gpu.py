"""GPU parity of the 14 drop-in ops (qsdvr_b200.qsdvr) against the reference's outputs:
the committed golden vectors, the reference build run live (oracle/_ref), and the oracle.

Bars: sample counts, offsets and cell indices bit-exact; float outputs within 1e-5
absolute (images) / 1e-6 relative (per-op values); gradients within 1e-4 relative."""
import numpy as np
import pytest
import torch

import oracle.oracle as O
from conftest import camera_from_record, oracle_camera, rel_err

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _t(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a)).to(DEV)
    return t if dtype is None else t.to(dtype)


@pytest.fixture(scope="module")
def qs():
    from qsdvr_b200 import _lib, qsdvr

    _lib.lib()
    return qsdvr


@pytest.fixture(scope="module")
def ref():
    from oracle.build_ref import load_reference

    r = load_reference()
    if r is None:
        pytest.skip("reference build (oracle/_ref) not present")
    return r


def _raycut_mine(qs, args, mask, interval):
    P = args.pixelCount
    rays = torch.zeros((P, 4), dtype=torch.int32, device=DEV)
    origin = torch.zeros((P, 3), device=DEV)
    direction = torch.zeros((P, 3), device=DEV)
    qs.RayCut(args, torch.from_numpy(np.asarray(mask, bool)), rays, origin, direction, interval)
    return rays, origin, direction


def _points_mine(qs, args, rays, origin, direction, interval, R):
    S, M = args.sdfCount, args.renderCount
    out = dict(sdfPointList=torch.zeros((S, 3), device=DEV), sdfIndexList=torch.zeros(S, dtype=torch.int32, device=DEV),
               renderPointList=torch.zeros((M, 3), device=DEV),
               renderIndexList=torch.zeros(M, dtype=torch.int32, device=DEV), viewDirList=torch.zeros((M, 3), device=DEV))
    qs.GenerateRayPoints(args, out["sdfPointList"], out["sdfIndexList"], out["renderPointList"], out["renderIndexList"],
                         out["viewDirList"], rays, origin, direction, interval, R)
    return out


# ------------------------------------------------------------------------ ray generation

@pytest.mark.parametrize("case", [0, 1, 2])
def test_raycut_bit_exact_vs_golden(qs, golden_raygen, case):
    g = golden_raygen
    args = camera_from_record(g[f"c{case}_camera"])
    interval, R = g[f"c{case}_params"]
    rays, origin, direction = _raycut_mine(qs, args, g[f"c{case}_mask"], float(interval))
    np.testing.assert_array_equal(rays.cpu().numpy(), g[f"c{case}_rays_all"])
    np.testing.assert_array_equal(direction.cpu().numpy(), g[f"c{case}_dir_all"])
    np.testing.assert_array_equal(origin.cpu().numpy(), g[f"c{case}_origin_all"])
    assert (args.sdfCount, args.renderCount) == tuple(g[f"c{case}_totals"])
    m = torch.from_numpy(g[f"c{case}_mask"]).to(DEV)
    pts = _points_mine(qs, args, rays[m].contiguous(), origin[m].contiguous(), direction[m].contiguous(),
                       float(interval), int(R))
    for k, v in pts.items():
        np.testing.assert_array_equal(v.cpu().numpy(), g[f"c{case}_{k}"], err_msg=k)


@pytest.mark.parametrize("size,interval,R", [(100, 4 / 64, 64), (800, 4 / 256, 256), (400, 4 / 512, 384)])
def test_raygen_bit_exact_vs_reference_live(qs, ref, size, interval, R):
    """Full-size cameras of the benchmark configs: every count, offset, direction, origin,
    sample point and cell index identical to the reference run on the same GPU."""
    from qsdvr_b200 import scenes
    from tests.golden.make_golden import run_raygen

    f = 1111.1 * size / 800
    for pos in [(0.4, -4.0, 0.3), (2.8, 2.1, 1.9)]:
        cam = scenes.look_at(pos, size, size, f, 2.0, 6.0)
        rng = np.random.default_rng(size)
        mask = rng.random(size * size) < 0.9
        want = run_raygen(ref, cam, mask, interval, R)
        rays, origin, direction = _raycut_mine(qs, cam, mask, interval)
        np.testing.assert_array_equal(rays.cpu().numpy(), want["rays_all"])
        np.testing.assert_array_equal(direction.cpu().numpy(), want["dir_all"])
        np.testing.assert_array_equal(origin.cpu().numpy(), want["origin_all"])
        m = torch.from_numpy(mask).to(DEV)
        pts = _points_mine(qs, cam, rays[m].contiguous(), origin[m].contiguous(), direction[m].contiguous(), interval, R)
        for k, v in pts.items():
            np.testing.assert_array_equal(v.cpu().numpy(), want[k], err_msg=k)


def test_raygen_matches_c_oracle(qs):
    from qsdvr_b200 import scenes

    cam = scenes.look_at((-3.0, 2.2, 1.4), 200, 150, 230.0, 2.0, 6.0)
    mask = np.random.default_rng(1).random(200 * 150) < 0.8
    rays, origin, direction = _raycut_mine(qs, cam, mask, 4 / 256)
    orays, oo, od, S, M = O.ray_cut(oracle_camera(cam), mask, 4 / 256)
    np.testing.assert_array_equal(rays.cpu().numpy().view(np.uint32), orays)
    np.testing.assert_array_equal(direction.cpu().numpy(), od)
    assert (cam.sdfCount, cam.renderCount) == (S, M)


# ------------------------------------------------------------------------ numeric ops vs golden

def test_quadric_ops_vs_golden(qs, golden_ops):
    g = golden_ops
    grid, pts, idx = _t(g["q_grid7"]), _t(g["q_points"]), _t(g["q_index"])
    S = pts.shape[0]
    sdf = torch.empty(S, device=DEV)
    qs.SampleSDFForward(sdf, grid, pts, idx, 8.0)
    assert rel_err(sdf.cpu(), g["q_sdf"]) < 1e-6
    nrm = torch.empty((S, 3), device=DEV)
    qs.SampleNormalForward(nrm, grid, pts, idx)
    assert rel_err(nrm.cpu(), g["q_normal"]) < 1e-6
    gs = torch.zeros_like(grid)
    qs.SampleSDFBackward(_t(g["q_gout1"]), grid, pts, idx, gs, 8.0)
    assert rel_err(gs.cpu(), g["q_sdf_grad"]) < 1e-5
    gn = torch.zeros_like(grid)
    qs.SampleNormalBackward(_t(g["q_gout3"]), grid, pts, idx, gn)
    assert rel_err(gn.cpu(), g["q_normal_grad"]) < 1e-5


def test_layer_to_grid_vs_golden(qs, golden_ops):
    g = golden_ops
    R = g["l_x"].shape[0]
    out = torch.empty((R, R, R, 7), device=DEV)
    qs.LayerToGridForward(out, *(torch.from_numpy(g[k]) for k in ("l_x", "l_y", "l_z", "l_offset")))
    assert rel_err(out.cpu(), g["l_grid7"]) < 1e-6
    bx, by, bz, bo = torch.empty(R), torch.empty(R), torch.empty(R), torch.empty(4)
    qs.LayerToGridBackward(_t(g["l_grad7"]), bx, by, bz, bo)
    for a, b in ((bx, "l_gx"), (by, "l_gy"), (bz, "l_gz"), (bo[:3], "l_goffset3")):
        assert rel_err(a, g[b]) < 1e-5, b


def test_layer_to_grid_large_vs_oracle(qs):
    R = 96
    gen = torch.Generator().manual_seed(3)
    x, y, z = (torch.rand(R, generator=gen) - 0.5 for _ in range(3))
    off = torch.rand(4, generator=gen)
    out = torch.empty((R, R, R, 7), device=DEV)
    qs.LayerToGridForward(out, x, y, z, off)
    want = O.layer_to_grid(x.double(), y.double(), z.double(), off.double())
    assert rel_err(out.cpu(), want) < 1e-5
    g7 = torch.rand((R, R, R, 7), generator=gen) - 0.5
    bx, by, bz, bo = torch.empty(R), torch.empty(R), torch.empty(R), torch.empty(4)
    qs.LayerToGridBackward(g7.to(DEV), bx, by, bz, bo)
    wx, wy, wz, wo = O.layer_to_grid_backward(g7.double())
    for a, b in ((bx, wx), (by, wy), (bz, wz), (bo, wo)):
        assert rel_err(a, b) < 1e-4


def test_grid_interpolation_vs_golden(qs, golden_ops):
    g = golden_ops
    data, pts, idx = _t(g["i_data"]), _t(g["i_points"]), _t(g["i_index"])
    reso = int(g["i_reso"])
    out = torch.empty((pts.shape[0], 32), device=DEV)
    qs.GridInterpolationForward(data, pts, idx, out, reso)
    assert rel_err(out.cpu(), g["i_out"]) < 1e-6
    gd = torch.zeros_like(data)
    qs.GridInterpolationBackward(gd, pts, idx, _t(g["i_gout"]), reso)
    assert rel_err(gd.cpu(), g["i_grad"]) < 1e-5


def test_shader_compat_vs_golden(qs, golden_ops):
    g = golden_ops
    n, v, d = _t(g["s_normal"]), _t(g["s_view"]), _t(g["s_data"])
    N = n.shape[0]
    out, spec = torch.empty((N, 3), device=DEV), torch.empty((N, 3), device=DEV)
    qs.ShaderForward(out, n, v, d, spec)
    assert rel_err(out.cpu(), g["s_out"]) < 1e-6
    assert rel_err(spec.cpu(), g["s_spec"]) < 1e-6
    ng, dg = torch.empty((N, 3), device=DEV), torch.empty((N, 32), device=DEV)
    qs.ShaderBackward(_t(g["s_gout"]), n, v, d, spec, ng, dg)
    assert rel_err(ng.cpu(), g["s_ngrad"]) < 1e-5
    assert rel_err(dg.cpu(), g["s_dgrad"]) < 1e-5


def test_shader_fixed_vs_oracle(qs, golden_ops):
    g = golden_ops
    n, v, d = _t(g["s_normal"]), _t(g["s_view"]), _t(g["s_data"])
    N = n.shape[0]
    out, spec = torch.empty((N, 3), device=DEV), torch.empty((N, 3), device=DEV)
    qs.ShaderForward(out, n, v, d, spec, mode="fixed")
    nd = torch.tensor(g["s_normal"], dtype=torch.float64, requires_grad=True)
    dd = torch.tensor(g["s_data"], dtype=torch.float64, requires_grad=True)
    rgb, _ = O.shader(nd, torch.tensor(g["s_view"], dtype=torch.float64), dd, compat=False)
    assert rel_err(out.cpu(), rgb.detach()) < 1e-6
    go = torch.tensor(g["s_gout"], dtype=torch.float64)
    wn, wd = torch.autograd.grad(rgb, (nd, dd), go)
    ng, dg = torch.empty((N, 3), device=DEV), torch.empty((N, 32), device=DEV)
    qs.ShaderBackward(_t(g["s_gout"]), n, v, d, spec, ng, dg, mode="fixed")
    assert rel_err(ng.cpu(), wn) < 1e-5
    assert rel_err(dg.cpu(), wd) < 1e-5


@pytest.mark.parametrize("kk", [0, 1])
def test_ray_aggregate_vs_golden(qs, golden_ops, kk):
    g = golden_ops
    k = float(g[f"a{kk}_k"])
    rays, rgb, sdf = _t(g["a_rays"]), _t(g["a_rgb"]), _t(g["a_sdf"])
    N, M, S = rays.shape[0], rgb.shape[0], sdf.shape[0]
    out, al, tl = torch.empty((N, 3), device=DEV), torch.empty(M, device=DEV), torch.empty(M, device=DEV)
    qs.RayAggregateForward(out, rgb, sdf, rays, al, tl, k)
    assert np.abs(out.cpu().numpy() - g[f"a{kk}_out"]).max() < 1e-5
    assert np.abs(al.cpu().numpy() - g[f"a{kk}_alpha"]).max() < 1e-6
    assert np.abs(tl.cpu().numpy() - g[f"a{kk}_T"]).max() < 1e-5
    rg, sg = torch.empty((M, 3), device=DEV), torch.empty(S, device=DEV)
    qs.RayAggregateBackward(_t(g["a_gout"]), rgb, sdf, rays, _t(g[f"a{kk}_alpha"]), _t(g[f"a{kk}_T"]), rg, sg, k)
    assert rel_err(rg.cpu(), g[f"a{kk}_rgb_grad"]) < 1e-4
    assert rel_err(sg.cpu(), g[f"a{kk}_sdf_grad"]) < 1e-4


# ------------------------------------------------------------------------ pipeline

def _chain(qs, grid7, data, inp, R, k, target, mode="compat"):
    """The RenderGrid op chain through the drop-in module (forward + MSE backward)."""
    S, M, N = inp["sdfPointList"].shape[0], inp["renderPointList"].shape[0], inp["rayList"].shape[0]
    sdf = torch.empty(S, device=DEV)
    qs.SampleSDFForward(sdf, grid7, inp["sdfPointList"], inp["sdfIndexList"], float(R))
    nrm = torch.empty((M, 3), device=DEV)
    qs.SampleNormalForward(nrm, grid7, inp["renderPointList"], inp["renderIndexList"])
    dl = torch.empty((M, 32), device=DEV)
    qs.GridInterpolationForward(data, inp["renderPointList"], inp["renderIndexList"], dl, R + 1)
    rgb, spec = torch.empty((M, 3), device=DEV), torch.empty((M, 3), device=DEV)
    qs.ShaderForward(rgb, nrm, inp["viewDirList"], dl, spec, mode=mode)
    img = torch.empty((N, 3), device=DEV)
    al, tl = torch.empty(M, device=DEV), torch.empty(M, device=DEV)
    qs.RayAggregateForward(img, rgb, sdf, inp["rayList"], al, tl, k)
    gimg = ((2.0 / img.numel()) * (img - target)).contiguous()
    grgb, gsdf = torch.empty((M, 3), device=DEV), torch.empty(S, device=DEV)
    qs.RayAggregateBackward(gimg, rgb, sdf, inp["rayList"], al, tl, grgb, gsdf, k)
    gn, gd = torch.empty((M, 3), device=DEV), torch.empty((M, 32), device=DEV)
    qs.ShaderBackward(grgb, nrm, inp["viewDirList"], dl, spec, gn, gd, mode=mode)
    gdata = torch.zeros_like(data)
    qs.GridInterpolationBackward(gdata, inp["renderPointList"], inp["renderIndexList"], gd, R + 1)
    ggrid = torch.zeros_like(grid7)
    qs.SampleNormalBackward(gn, grid7, inp["renderPointList"], inp["renderIndexList"], ggrid)
    qs.SampleSDFBackward(gsdf, grid7, inp["sdfPointList"], inp["sdfIndexList"], ggrid, float(R))
    return img, ggrid, gdata


def test_pipeline_vs_golden(qs, golden_pipeline):
    g = golden_pipeline
    R, k, _ = g["params"]
    R = int(R)
    inp = {kk: _t(g["in_" + kk]) for kk in ("sdfPointList", "sdfIndexList", "renderPointList", "renderIndexList",
                                             "viewDirList")}
    inp["rayList"] = _t(g["in_rays"])
    img, gg, gd = _chain(qs, _t(g["grid7"]), _t(g["data"]), inp, R, float(k), _t(g["target"]))
    assert np.abs(img.cpu().numpy() - g["image"]).max() < 1e-5
    assert rel_err(gg.cpu(), g["grid7_grad"]) < 1e-4
    assert rel_err(gd.cpu(), g["data_grad"]) < 1e-4


def test_pipeline_config1_vs_reference_live(qs, ref):
    """Config-1 scene (64^3 grid, 100x100 camera, 64 samples/ray) through the drop-in chain
    and through the reference build on the same inputs."""
    from qsdvr_b200 import scenes
    from tests.golden.make_golden import reference_render, run_raygen

    R, k, interval = 64, 10.0, 4.0 / 64
    cam = scenes.look_at((0.0, -4.0, 0.0), 100, 100, 138.9, 2.0, 6.0)
    rg = run_raygen(ref, cam, np.ones(100 * 100, bool), interval, R)
    inp = {kk: _t(rg[kk]) for kk in ("sdfPointList", "sdfIndexList", "renderPointList", "renderIndexList",
                                      "viewDirList")}
    inp["rayList"] = _t(rg["rays"])
    grid7 = scenes.sphere_grid(R).reshape(-1, 7).to(DEV)
    data = scenes.appearance(R).to(DEV)
    target = torch.rand((rg["rays"].shape[0], 3), generator=torch.Generator().manual_seed(0)).to(DEV)
    want = reference_render(ref, grid7, data, inp, R, k, target)
    got = _chain(qs, grid7, data, inp, R, k, target)
    assert np.abs(got[0].cpu().numpy() - want[0].cpu().numpy()).max() < 1e-5
    assert rel_err(got[1].cpu(), want[1].cpu()) < 1e-4
    assert rel_err(got[2].cpu(), want[2].cpu()) < 1e-4


def test_render_grid_module_vs_reference_chain(qs, ref):
    """qsdvr_b200.render.RenderGrid (separable layers, autograd) against the reference's
    own ops chained exactly as models/render.py does."""
    from qsdvr_b200 import scenes
    from qsdvr_b200.render import RenderGrid
    from tests.golden.make_golden import run_raygen

    R, k, interval = 32, 0.5, 4.0 / 64
    cam = scenes.look_at((1.0, -3.8, 0.9), 64, 64, 90.0, 2.0, 6.0)
    rg = run_raygen(ref, cam, np.ones(64 * 64, bool), interval, R)
    inp = {kk: _t(rg[kk]) for kk in ("sdfPointList", "sdfIndexList", "renderPointList", "renderIndexList",
                                      "viewDirList")}
    inp["rayList"] = _t(rg["rays"])
    model = RenderGrid(R, k)
    with torch.no_grad():
        gen = torch.Generator().manual_seed(5)
        model.quadricGrid.xLayer.add_(0.01 * torch.randn(R, generator=gen))
        model.renderData.add_(0.05 * torch.randn(model.renderData.shape, generator=gen).to(DEV))
    img = model(inp)
    loss = img.square().mean()
    loss.backward()
    # reference chain
    grid = torch.empty((R, R, R, 7), device=DEV)
    ref.LayerToGridForward(grid, model.quadricGrid.xLayer.detach().clone(), model.quadricGrid.yLayer.detach().clone(),
                           model.quadricGrid.zLayer.detach().clone(), model.quadricGrid.offset.detach().clone())
    from tests.golden.make_golden import reference_render

    data = model.renderData.detach().reshape(-1, 32).contiguous()
    want_img, ggrid, gdata = reference_render(ref, grid.reshape(-1, 7), data, inp, R, k,
                                              torch.zeros_like(img))
    assert np.abs(img.detach().cpu().numpy() - want_img.cpu().numpy()).max() < 1e-5
    assert rel_err(model.renderData.grad.reshape(-1, 32).cpu(), gdata.cpu()) < 1e-4
    from oracle.build_ref import reference_layer_to_grid_backward

    bx, by, bz, bo = reference_layer_to_grid_backward(ref, ggrid.reshape(R, R, R, 7), R)
    assert rel_err(model.quadricGrid.xLayer.grad, bx) < 1e-4
    assert rel_err(model.quadricGrid.zLayer.grad, bz) < 1e-4
    assert rel_err(model.quadricGrid.offset.grad[:3], bo) < 1e-4
    # offset[3]: the reference never writes it; ours is the sum of all a6 gradients
    assert abs(model.quadricGrid.offset.grad[3].item() - ggrid.reshape(-1, 7)[:, 6].sum().item()) < 1e-4 * max(
        1.0, ggrid.reshape(-1, 7)[:, 6].abs().sum().item())


def test_bad_indices_flag_error_without_fault(qs):
    from qsdvr_b200 import _lib

    _lib.device_error()  # clear
    grid = torch.zeros((8 ** 3, 7), device=DEV)
    pts = torch.zeros((4, 3), device=DEV)
    idx = torch.tensor([0, 511, 512, -3], dtype=torch.int32, device=DEV)
    out = torch.full((4,), 7.0, device=DEV)
    qs.SampleSDFForward(out, grid, pts, idx, 8.0)
    assert _lib.device_error() & _lib.DEVERR_INDEX
    assert out[2].item() == 0.0 and out[3].item() == 0.0
    data = torch.zeros((9 ** 3, 32), device=DEV)
    dl = torch.empty((4, 32), device=DEV)
    qs.GridInterpolationForward(data, pts, torch.tensor([0, 700, 1, 2], dtype=torch.int32, device=DEV), dl, 9)
    assert _lib.device_error() & _lib.DEVERR_INDEX
    assert _lib.device_error() == 0
