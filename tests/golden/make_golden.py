"""Generate the golden vectors in tests/golden/ by running the REFERENCE on a B200.

The reference (QSDVR's own CUDA extension) is compiled from its sources by
oracle/build_ref.py into oracle/_ref/; this script imports that build, feeds it seeded
inputs and saves inputs and outputs as compressed .npz fixtures:

  raygen.npz    RayCut + GenerateRayPoints on three seeded cameras (counts, offsets,
                origins, directions, sample points, cell indices)
  ops.npz       each of the 12 numeric ops on seeded random inputs
  pipeline.npz  the RenderGrid forward/backward chain (dense quadric grid) on a small
                seeded scene: image and gradients of the SDF grid and appearance grid

Inputs are chosen so that every reference kernel stays in bounds: cell indices < R^3,
render counts = sdf counts - 1, ray counts 0 or >= 2, and the offset tensor handed to
LayerToGridBackward is R+3 floats long (it copies R floats into offset[3:]).  That copy
reads R floats from a 1-float device buffer and fails (cudaErrorInvalidValue), so the
reference never writes the offset[3] gradient; only offset[0:3] is recorded.

Usage (GPU box):  python tests/golden/make_golden.py [--out DIR] [--big]
``--big`` additionally writes raygen_big.npz (two 400x400 cameras) for offline analysis.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.build_ref import load_reference, reference_layer_to_grid_backward  # noqa: E402
from qsdvr_b200 import scenes  # noqa: E402

DEV = "cuda"


def ref_camera(ref, cam):
    a = ref.CameraArgs()
    a.width, a.height = cam.width, cam.height
    a.rotation = [float(v) for v in cam.rotation]
    a.translation = [float(v) for v in cam.translation]
    a.fx, a.fy, a.cx, a.cy = cam.fx, cam.fy, cam.cx, cam.cy
    a.near, a.far = cam.near, cam.far
    a.pixelCount = cam.width * cam.height
    return a


def run_raygen(ref, cam, mask: np.ndarray, interval: float, reso: int):
    """RayCut over all pixels then GenerateRayPoints over the masked rays (datasets/utils.py:42-56, :16-40)."""
    a = ref_camera(ref, cam)
    P = a.pixelCount
    rays = torch.zeros((P, 4), dtype=torch.int32, device=DEV)
    origin = torch.zeros((P, 3), dtype=torch.float32, device=DEV)
    direction = torch.zeros((P, 3), dtype=torch.float32, device=DEV)
    m = torch.from_numpy(mask.astype(bool))
    ref.RayCut(a, m, rays, origin, direction, interval)
    torch.cuda.synchronize()
    out = dict(rays_all=rays.cpu().numpy(), origin_all=origin.cpu().numpy(), dir_all=direction.cpu().numpy(),
               totals=np.array([a.sdfCount, a.renderCount], np.int64))
    mr = rays[m.to(DEV)].contiguous()
    mo = origin[m.to(DEV)].contiguous()
    md = direction[m.to(DEV)].contiguous()
    S, M = a.sdfCount, a.renderCount
    sp = torch.zeros((S, 3), dtype=torch.float32, device=DEV)
    si = torch.zeros(S, dtype=torch.int32, device=DEV)
    rp = torch.zeros((M, 3), dtype=torch.float32, device=DEV)
    ri = torch.zeros(M, dtype=torch.int32, device=DEV)
    vd = torch.zeros((M, 3), dtype=torch.float32, device=DEV)
    ref.GenerateRayPoints(a, sp, si, rp, ri, vd, mr, mo, md, interval, reso)
    torch.cuda.synchronize()
    out.update(rays=mr.cpu().numpy(), origin=mo.cpu().numpy(), dir=md.cpu().numpy(), sdfPointList=sp.cpu().numpy(),
               sdfIndexList=si.cpu().numpy(), renderPointList=rp.cpu().numpy(), renderIndexList=ri.cpu().numpy(),
               viewDirList=vd.cpu().numpy())
    return out


def camera_record(cam):
    return np.array([cam.width, cam.height, *cam.rotation, *cam.translation, cam.fx, cam.fy, cam.cx, cam.cy, cam.near,
                     cam.far], np.float64)


RAYGEN_CASES = [
    # (position, width, height, focal, near, far, interval, reso, mask density)
    ((0.3, -4.0, 0.7), 64, 48, 80.0, 2.0, 6.0, 4.0 / 64, 16, 0.7),
    ((2.5, 2.5, 2.2), 64, 64, 88.9, 2.0, 6.0, 4.0 / 64, 64, 1.0),
    ((-1.0, 0.5, 4.03), 40, 30, 55.5, 2.0, 6.0, 4.0 / 256, 48, 0.9),
]


def make_raygen(ref, out_dir, big=False):
    rng = np.random.default_rng(0)
    rec = {}
    for c, (pos, w, h, f, n, fa, iv, R, dens) in enumerate(RAYGEN_CASES):
        cam = scenes.look_at(pos, w, h, f, n, fa)
        mask = rng.random(w * h) < dens
        o = run_raygen(ref, cam, mask, iv, R)
        rec[f"c{c}_camera"] = camera_record(cam)
        rec[f"c{c}_mask"] = mask
        rec[f"c{c}_params"] = np.array([iv, R], np.float64)
        for k, v in o.items():
            rec[f"c{c}_{k}"] = v
    np.savez_compressed(os.path.join(out_dir, "raygen.npz"), **rec)
    if big:
        rec = {}
        for c, pos in enumerate([(0.7, -3.9, 1.1), (-2.9, -2.0, 2.0)]):
            cam = scenes.look_at(pos, 400, 400, 555.5, 2.0, 6.0)
            mask = np.ones(400 * 400, bool)
            o = run_raygen(ref, cam, mask, 4.0 / 256, 256)
            rec[f"c{c}_camera"] = camera_record(cam)
            for k in ("rays_all", "origin_all", "dir_all", "totals", "sdfIndexList", "renderIndexList"):
                rec[f"c{c}_{k}"] = o[k]
        np.savez_compressed(os.path.join(out_dir, "raygen_big.npz"), **rec)


def make_ops(ref, out_dir):
    g = torch.Generator().manual_seed(1234)
    rnd = lambda *s: torch.rand(*s, generator=g)  # noqa: E731
    rec = {}
    # --- quadric grid ops, R = 8
    R, S = 8, 3000
    grid7 = rnd(R ** 3, 7) * 2 - 1
    grid7[:, 3:6] += torch.sign(grid7[:, 3:6]) * 3.0  # |2 a_k u_k + a_{k+3}| >= 1
    pts = rnd(S, 3) * 2 - 1
    idx = torch.randint(0, R ** 3, (S,), generator=g, dtype=torch.int32)
    gout1 = rnd(S) - 0.5
    gout3 = rnd(S, 3) - 0.5
    dg, dp, di = grid7.to(DEV), pts.to(DEV), idx.to(DEV)
    sdf = torch.empty(S, device=DEV)
    ref.SampleSDFForward(sdf, dg, dp, di, float(R))
    nrm = torch.empty((S, 3), device=DEV)
    ref.SampleNormalForward(nrm, dg, dp, di)
    gs = torch.zeros((R ** 3, 7), device=DEV)
    ref.SampleSDFBackward(gout1.to(DEV), dg, dp, di, gs, float(R))
    gn = torch.zeros((R ** 3, 7), device=DEV)
    ref.SampleNormalBackward(gout3.to(DEV), dg, dp, di, gn)
    rec.update(q_grid7=grid7.numpy(), q_points=pts.numpy(), q_index=idx.numpy(), q_gout1=gout1.numpy(),
               q_gout3=gout3.numpy(), q_sdf=sdf.cpu().numpy(), q_normal=nrm.cpu().numpy(),
               q_sdf_grad=gs.cpu().numpy(), q_normal_grad=gn.cpu().numpy())
    # --- layer to grid, R = 8
    xl, yl, zl = rnd(R) - 0.5, rnd(R) - 0.5, rnd(R) - 0.5
    off = rnd(4) * 2 - 1
    lg = torch.empty((R, R, R, 7), device=DEV)
    ref.LayerToGridForward(lg, xl, yl, zl, off)
    g7 = rnd(R, R, R, 7) - 0.5
    bx, by, bz, boff = reference_layer_to_grid_backward(ref, g7.to(DEV), R)
    rec.update(l_x=xl.numpy(), l_y=yl.numpy(), l_z=zl.numpy(), l_offset=off.numpy(), l_grid7=lg.cpu().numpy(),
               l_grad7=g7.numpy(), l_gx=bx.numpy(), l_gy=by.numpy(), l_gz=bz.numpy(), l_goffset3=boff.numpy())
    # --- grid interpolation: vertex grid (R+1)^3 addressed with cell indices of stride R
    V = (R + 1) ** 3
    data = rnd(V, 32) * 2 - 1
    M = 1000
    ipts = rnd(M, 3) * 2 - 1
    iidx = torch.randint(0, R ** 3, (M,), generator=g, dtype=torch.int32)
    igo = rnd(M, 32) - 0.5
    iout = torch.empty((M, 32), device=DEV)
    ref.GridInterpolationForward(data.to(DEV), ipts.to(DEV), iidx.to(DEV), iout, R + 1)
    igrad = torch.zeros((V, 32), device=DEV)
    ref.GridInterpolationBackward(igrad, ipts.to(DEV), iidx.to(DEV), igo.to(DEV), R + 1)
    rec.update(i_data=data.numpy(), i_points=ipts.numpy(), i_index=iidx.numpy(), i_gout=igo.numpy(),
               i_out=iout.cpu().numpy(), i_grad=igrad.cpu().numpy(), i_reso=np.array(R + 1))
    # --- shader
    N = 1000
    n = torch.nn.functional.normalize(rnd(N, 3) - 0.5, dim=1)
    v = torch.nn.functional.normalize(rnd(N, 3) - 0.5, dim=1)
    sd = rnd(N, 32)
    sgo = rnd(N, 3) - 0.5
    sout, sspec = torch.empty((N, 3), device=DEV), torch.empty((N, 3), device=DEV)
    ref.ShaderForward(sout, n.to(DEV), v.to(DEV), sd.to(DEV), sspec)
    sng, sdg = torch.empty((N, 3), device=DEV), torch.empty((N, 32), device=DEV)
    ref.ShaderBackward(sgo.to(DEV), n.to(DEV), v.to(DEV), sd.to(DEV), sspec, sng, sdg)
    rec.update(s_normal=n.numpy(), s_view=v.numpy(), s_data=sd.numpy(), s_gout=sgo.numpy(), s_out=sout.cpu().numpy(),
               s_spec=sspec.cpu().numpy(), s_ngrad=sng.cpu().numpy(), s_dgrad=sdg.cpu().numpy())
    # --- ray aggregate: counts 0 or >= 2, render = sdf - 1, rays longer than a warp
    counts = np.array([0, 2, 3, 5, 0, 33, 40, 70, 2, 129, 17, 0, 64, 65, 31, 32, 200], np.int64)
    rays = np.zeros((counts.size, 4), np.int32)
    so = ro = 0
    for i, c in enumerate(counts):
        rays[i] = (c, so, max(c - 1, 0), ro)
        so += c
        ro += max(c - 1, 0)
    sdfv = (rnd(so) - 0.45) * 0.6
    rgb = rnd(ro, 3)
    rgo = rnd(counts.size, 3) - 0.5
    for kk, k in enumerate((5.0, 50.0)):
        out = torch.empty((counts.size, 3), device=DEV)
        al, tl = torch.empty(ro, device=DEV), torch.empty(ro, device=DEV)
        dr = torch.from_numpy(rays).to(DEV)
        ref.RayAggregateForward(out, rgb.to(DEV), sdfv.to(DEV), dr, al, tl, k)
        rg, sg = torch.empty((ro, 3), device=DEV), torch.empty(so, device=DEV)
        ref.RayAggregateBackward(rgo.to(DEV), rgb.to(DEV), sdfv.to(DEV), dr, al, tl, rg, sg, k)
        rec.update({f"a{kk}_k": np.array(k), f"a{kk}_out": out.cpu().numpy(), f"a{kk}_alpha": al.cpu().numpy(),
                    f"a{kk}_T": tl.cpu().numpy(), f"a{kk}_rgb_grad": rg.cpu().numpy(),
                    f"a{kk}_sdf_grad": sg.cpu().numpy()})
    rec.update(a_rays=rays, a_sdf=sdfv.numpy(), a_rgb=rgb.numpy(), a_gout=rgo.numpy())
    torch.cuda.synchronize()
    np.savez_compressed(os.path.join(out_dir, "ops.npz"), **rec)


def reference_render(ref, grid7, data, inp, R, k, target):
    """The RenderGrid chain (models/render.py:225-234) on a dense grid, forward + MSE backward."""
    S = inp["sdfPointList"].shape[0]
    M = inp["renderPointList"].shape[0]
    N = inp["rayList"].shape[0]
    sdf = torch.empty(S, device=DEV)
    ref.SampleSDFForward(sdf, grid7, inp["sdfPointList"], inp["sdfIndexList"], float(R))
    nrm = torch.empty((M, 3), device=DEV)
    ref.SampleNormalForward(nrm, grid7, inp["renderPointList"], inp["renderIndexList"])
    dl = torch.empty((M, 32), device=DEV)
    ref.GridInterpolationForward(data, inp["renderPointList"], inp["renderIndexList"], dl, R + 1)
    rgb, spec = torch.empty((M, 3), device=DEV), torch.empty((M, 3), device=DEV)
    ref.ShaderForward(rgb, nrm, inp["viewDirList"], dl, spec)
    img = torch.empty((N, 3), device=DEV)
    al, tl = torch.empty(M, device=DEV), torch.empty(M, device=DEV)
    ref.RayAggregateForward(img, rgb, sdf, inp["rayList"], al, tl, k)
    gimg = (2.0 / img.numel()) * (img - target)
    grgb, gsdf = torch.empty((M, 3), device=DEV), torch.empty(S, device=DEV)
    ref.RayAggregateBackward(gimg.contiguous(), rgb, sdf, inp["rayList"], al, tl, grgb, gsdf, k)
    gn, gd = torch.empty((M, 3), device=DEV), torch.empty((M, 32), device=DEV)
    ref.ShaderBackward(grgb, nrm, inp["viewDirList"], dl, spec, gn, gd)
    gdata = torch.zeros_like(data)
    ref.GridInterpolationBackward(gdata, inp["renderPointList"], inp["renderIndexList"], gd, R + 1)
    ggrid = torch.zeros_like(grid7)
    ref.SampleNormalBackward(gn, grid7, inp["renderPointList"], inp["renderIndexList"], ggrid)
    ref.SampleSDFBackward(gsdf, grid7, inp["sdfPointList"], inp["sdfIndexList"], ggrid, float(R))
    torch.cuda.synchronize()
    return img, ggrid, gdata


def make_pipeline(ref, out_dir):
    R, k, interval = 16, 10.0, 4.0 / 64  # k large enough for opaque surfaces, small enough that alpha < 1
    cam = scenes.look_at((0.4, -4.0, 0.6), 40, 32, 55.0, 2.0, 6.0)
    mask = np.ones(cam.width * cam.height, bool)
    rg = run_raygen(ref, cam, mask, interval, R)
    inp = {kk: torch.from_numpy(rg[kk]).to(DEV) for kk in ("sdfPointList", "sdfIndexList", "renderPointList",
                                                            "renderIndexList", "viewDirList")}
    inp["rayList"] = torch.from_numpy(rg["rays"]).to(DEV)
    grid7 = scenes.sphere_grid(R, 0.5, 0.01, seed=0).reshape(-1, 7).to(DEV)
    data = scenes.appearance(R, seed=0).to(DEV)
    gen = torch.Generator().manual_seed(7)
    target = torch.rand((rg["rays"].shape[0], 3), generator=gen).to(DEV)
    img, ggrid, gdata = reference_render(ref, grid7, data, inp, R, k, target)
    rec = dict(camera=camera_record(cam), params=np.array([R, k, interval]), grid7=grid7.cpu().numpy(),
               data=data.cpu().numpy(), target=target.cpu().numpy(), image=img.cpu().numpy(),
               grid7_grad=ggrid.cpu().numpy(), data_grad=gdata.cpu().numpy())
    rec.update({f"in_{kk}": v for kk, v in rg.items() if kk in ("rays", "origin", "dir", "sdfPointList", "sdfIndexList",
                                                               "renderPointList", "renderIndexList", "viewDirList")})
    np.savez_compressed(os.path.join(out_dir, "pipeline.npz"), **rec)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    ap.add_argument("--big", action="store_true")
    a = ap.parse_args()
    ref = load_reference()
    if ref is None:
        raise SystemExit("oracle/_ref is not built (python oracle/build_ref.py)")
    os.makedirs(a.out, exist_ok=True)
    torch.manual_seed(0)
    make_raygen(ref, a.out, a.big)
    make_ops(ref, a.out)
    make_pipeline(ref, a.out)
    print("golden vectors written to", a.out)


if __name__ == "__main__":
    main()
