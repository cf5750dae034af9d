"""The oracle against the reference's own outputs (golden vectors made by running the
reference on a B200) and against itself (autograd vs the reference's backward formulas).
CPU only."""
import numpy as np
import pytest
import torch

import oracle.oracle as O
from conftest import camera_from_record, oracle_camera, rel_err



# ------------------------------------------------------------------------ ray generation

@pytest.mark.parametrize("case", [0, 1, 2])
def test_oracle_raycut_bit_exact(golden_raygen, case):
    g = golden_raygen
    args = camera_from_record(g[f"c{case}_camera"])
    interval, R = g[f"c{case}_params"]
    rays, origin, direction, S, M = O.ray_cut(oracle_camera(args), g[f"c{case}_mask"], float(interval))
    np.testing.assert_array_equal(rays.view(np.int32), g[f"c{case}_rays_all"])
    np.testing.assert_array_equal(direction, g[f"c{case}_dir_all"])
    np.testing.assert_array_equal(origin, g[f"c{case}_origin_all"])
    assert (S, M) == tuple(g[f"c{case}_totals"])


@pytest.mark.parametrize("case", [0, 1, 2])
def test_oracle_generate_points_bit_exact(golden_raygen, case):
    g = golden_raygen
    interval, R = g[f"c{case}_params"]
    out = O.generate_ray_points(g[f"c{case}_rays"].view(np.uint32), g[f"c{case}_origin"], g[f"c{case}_dir"],
                                float(interval), int(R))
    for k in ("sdfIndexList", "renderIndexList", "sdfPointList", "renderPointList", "viewDirList"):
        np.testing.assert_array_equal(out[k], g[f"c{case}_{k}"], err_msg=k)


# ------------------------------------------------------------------------ numeric ops

def test_oracle_quadric_ops(golden_ops):
    g = golden_ops
    grid = torch.tensor(g["q_grid7"], requires_grad=True)
    sdf = O.sample_sdf(grid, g["q_points"], g["q_index"], 8.0)
    assert rel_err(sdf.detach(), g["q_sdf"]) < 1e-6
    (gs,) = torch.autograd.grad(sdf, grid, torch.tensor(g["q_gout1"]))
    assert rel_err(gs, g["q_sdf_grad"]) < 1e-5
    nrm = O.sample_normal(grid, g["q_points"], g["q_index"])
    assert rel_err(nrm.detach(), g["q_normal"]) < 1e-6
    (gn,) = torch.autograd.grad(nrm, grid, torch.tensor(g["q_gout3"]))
    assert rel_err(gn, g["q_normal_grad"]) < 1e-5


def test_oracle_layer_to_grid(golden_ops):
    g = golden_ops
    out = O.layer_to_grid(*(torch.tensor(g[k]) for k in ("l_x", "l_y", "l_z", "l_offset")))
    assert rel_err(out, g["l_grid7"]) < 1e-6
    gx, gy, gz, go = O.layer_to_grid_backward(torch.tensor(g["l_grad7"]))
    for a, b in ((gx, "l_gx"), (gy, "l_gy"), (gz, "l_gz"), (go[:3], "l_goffset3")):
        assert rel_err(a, g[b]) < 1e-5, b


def test_oracle_grid_interpolation(golden_ops):
    g = golden_ops
    data = torch.tensor(g["i_data"], requires_grad=True)
    out = O.grid_interpolation(data, g["i_points"], g["i_index"], int(g["i_reso"]))
    assert rel_err(out.detach(), g["i_out"]) < 1e-6
    (gd,) = torch.autograd.grad(out, data, torch.tensor(g["i_gout"]))
    assert rel_err(gd, g["i_grad"]) < 1e-5


def test_oracle_shader_compat(golden_ops):
    g = golden_ops
    n, v, d = (torch.tensor(g[k]) for k in ("s_normal", "s_view", "s_data"))
    rgb, spec = O.shader(n, v, d, compat=True)
    assert rel_err(rgb, g["s_out"]) < 1e-6
    assert rel_err(spec, g["s_spec"]) < 1e-6
    ng, dg = O.shader_backward_reference(g["s_gout"], n, v, d, spec, compat=True)
    assert rel_err(ng, g["s_ngrad"]) < 1e-5
    assert rel_err(dg, g["s_dgrad"]) < 1e-5


@pytest.mark.parametrize("kk", [0, 1])
def test_oracle_ray_aggregate(golden_ops, kk):
    g = golden_ops
    k = float(g[f"a{kk}_k"])
    rgb, sdf = torch.tensor(g["a_rgb"]), torch.tensor(g["a_sdf"])
    color, alpha, T = O.ray_aggregate(rgb, sdf, g["a_rays"], k)
    assert np.abs(color.numpy() - g[f"a{kk}_out"]).max() < 1e-5
    assert np.abs(alpha.numpy() - g[f"a{kk}_alpha"]).max() < 1e-5
    assert np.abs(T.numpy() - g[f"a{kk}_T"]).max() < 1e-5
    rg, sg = O.ray_aggregate_backward_reference(g["a_gout"], rgb, sdf, g["a_rays"], g[f"a{kk}_alpha"], g[f"a{kk}_T"], k)
    assert rel_err(rg, g[f"a{kk}_rgb_grad"]) < 1e-4
    assert rel_err(sg, g[f"a{kk}_sdf_grad"]) < 1e-4


def test_oracle_pipeline(golden_pipeline):
    g = golden_pipeline
    R, k, _ = g["params"]
    R = int(R)
    inp = {kk: torch.from_numpy(g["in_" + kk]) for kk in ("sdfPointList", "sdfIndexList", "renderPointList",
                                                           "renderIndexList", "viewDirList")}
    inp["rayList"] = torch.from_numpy(g["in_rays"].astype(np.int64))
    grid = torch.tensor(g["grid7"], requires_grad=True)
    data = torch.tensor(g["data"], requires_grad=True)
    img = O.render(grid, data, inp, float(k), compat=True)
    assert np.abs(img.detach().numpy() - g["image"]).max() < 1e-5
    loss = ((img - torch.tensor(g["target"])) ** 2).mean()
    gg, gd = torch.autograd.grad(loss, (grid, data))
    assert rel_err(gg, g["grid7_grad"]) < 1e-4
    assert rel_err(gd, g["data_grad"]) < 1e-4


# ------------------------------------------------------------------------ self-consistency

def _aggregate_case(seed=0, k=20.0):
    rng = np.random.default_rng(seed)
    counts = [0, 2, 7, 40, 3]
    rays, so, ro = [], 0, 0
    for c in counts:
        rays.append((c, so, max(c - 1, 0), ro))
        so += c
        ro += max(c - 1, 0)
    rays = np.array(rays, np.int64)
    sdf = torch.tensor(rng.uniform(-0.2, 0.3, so), requires_grad=True)
    rgb = torch.tensor(rng.uniform(0, 1, (ro, 3)), requires_grad=True)
    gout = torch.tensor(rng.uniform(-1, 1, (len(counts), 3)))
    return rays, sdf, rgb, gout, k


def test_aggregate_reference_backward_is_autograd():
    rays, sdf, rgb, gout, k = _aggregate_case()
    color, alpha, T = O.ray_aggregate(rgb, sdf, rays, k)
    ga_rgb, ga_sdf = torch.autograd.grad(color, (rgb, sdf), gout)
    rg, sg = O.ray_aggregate_backward_reference(gout, rgb.detach(), sdf.detach(), rays, alpha, T, k)
    assert rel_err(rg, ga_rgb) < 1e-12
    assert rel_err(sg, ga_sdf) < 1e-12


def test_shader_fixed_backward_is_autograd():
    rng = np.random.default_rng(3)
    n = torch.nn.functional.normalize(torch.tensor(rng.normal(size=(50, 3))), dim=1).requires_grad_()
    v = torch.nn.functional.normalize(torch.tensor(rng.normal(size=(50, 3))), dim=1)
    d = torch.tensor(rng.uniform(0, 1, (50, 32)), requires_grad=True)
    rgb, spec = O.shader(n, v, d, compat=False)
    go = torch.tensor(rng.normal(size=(50, 3)))
    gn, gd = torch.autograd.grad(rgb, (n, d), go)
    ng, dg = O.shader_backward_reference(go, n.detach(), v, d.detach(), spec.detach(), compat=False)
    assert rel_err(ng, gn) < 1e-12
    assert rel_err(dg, gd) < 1e-12


def test_shader_compat_backward_differs_from_autograd():
    """Q1: in compat mode the reference's data gradient is NOT the gradient of its forward."""
    rng = np.random.default_rng(4)
    n = torch.nn.functional.normalize(torch.tensor(rng.normal(size=(50, 3))), dim=1)
    v = torch.nn.functional.normalize(torch.tensor(rng.normal(size=(50, 3))), dim=1)
    d = torch.tensor(rng.uniform(0, 1, (50, 32)), requires_grad=True)
    rgb, spec = O.shader(n, v, d, compat=True)
    go = torch.tensor(rng.normal(size=(50, 3)))
    (gd,) = torch.autograd.grad(rgb, d, go)
    _, dg = O.shader_backward_reference(go, n, v, d.detach(), spec.detach(), compat=True)
    assert rel_err(dg, gd) > 1e-3


def test_layer_to_grid_matches_dense_definition():
    rng = np.random.default_rng(5)
    R = 6
    x, y, z = (torch.tensor(rng.normal(size=R)) for _ in range(3))
    off = torch.tensor(rng.normal(size=4))
    g = O.layer_to_grid(x, y, z, off)
    # kernel/surface.cu:161-178 written as explicit loops
    def rec(a0, o):
        a3, a6 = [o], [0.0]
        for i in range(1, R):
            a3.append(2 * a0[i - 1] + 2 * a0[i] + a3[i - 1])
        for i in range(1, R):
            a6.append(3 * a0[i - 1] + a0[i] + 2 * a3[i - 1] + a6[i - 1])
        return a3, a6
    x3, x6 = rec(x.tolist(), off[0].item())
    y4, y6 = rec(y.tolist(), off[1].item())
    z5, z6 = rec(z.tolist(), off[2].item())
    for (zi, yi, xi) in [(0, 0, 0), (1, 2, 3), (5, 4, 0), (2, 5, 5)]:
        want = [x[xi], y[yi], z[zi], x3[xi], y4[yi], z5[zi], x6[xi] + y6[yi] + z6[zi] + off[3]]
        np.testing.assert_allclose(g[zi, yi, xi].numpy(), np.array([float(w) for w in want]), rtol=1e-12)


def test_raycut_counts_contiguous_and_offsets():
    """RayCut: masked counts < 2 are zeroed and offsets are an exclusive scan over masked pixels."""
    from qsdvr_b200 import scenes

    cam = scenes.look_at((0.2, -3.5, 1.0), 40, 30, 50.0, 2.0, 6.0)
    rng = np.random.default_rng(0)
    mask = rng.random(40 * 30) < 0.6
    rays, o, d, S, M = O.ray_cut(oracle_camera(cam), mask, 4 / 64)
    sc = np.where(mask, rays[:, 0], 0)
    assert not np.any((sc == 1))
    np.testing.assert_array_equal(rays[mask, 1], np.cumsum(sc[mask]) - sc[mask])
    rc = np.where(sc > 1, sc - 1, 0)
    np.testing.assert_array_equal(rays[mask, 3], np.cumsum(rc[mask]) - rc[mask])
    assert S == sc.sum() and M == rc.sum()


def test_bf16_cell_form_keeps_the_centre_sdf():
    """The bf16 cell form (oracle restatement of qsdvr_sdf_cells_bf16): a0..a5 are torch's
    round-to-nearest bf16, and the decoded cell's SDF at its centre, a6 / |a3..a5| / R, equals
    the fp32 master's to the 16 bits of the hi + lo pair, where a plain rounding misses it by
    up to 2^-8 relative."""
    import oracle.oracle as O
    from qsdvr_b200 import scenes

    g7 = scenes.procedural_grid(16, seed=2).reshape(-1, 7)
    g8 = np.zeros((g7.shape[0], 8), np.float32)
    g8[:, :7] = g7.numpy()
    bits = O.sdf_cells_bf16(g8)
    plain = torch.from_numpy(g8[:, :6]).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    assert np.array_equal(bits[:, :6], plain)
    dec = O.sdf_cells_decode(bits).double().numpy()
    m = g8.astype(np.float64)
    centre = m[:, 6] / np.linalg.norm(m[:, 3:6], axis=1)
    got = dec[:, 6] / np.linalg.norm(dec[:, 3:6], axis=1)
    rel = np.abs(got - centre) / np.abs(centre)
    assert rel.max() < 2.0 ** -16
    pl = torch.from_numpy(g8).to(torch.bfloat16).double().numpy()
    rel_plain = np.abs(pl[:, 6] / np.linalg.norm(pl[:, 3:6], axis=1) - centre) / np.abs(centre)
    assert rel_plain.max() > 2.0 ** -10
    # a plain-rounded copy (slot 7 = 0) decodes to a6 = bf16(a6)
    pb = torch.from_numpy(g8).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    assert np.array_equal(O.sdf_cells_decode(pb).numpy()[:, 6], pl[:, 6].astype(np.float32))
