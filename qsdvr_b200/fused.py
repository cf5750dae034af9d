"""Fused render path: one kernel per pass over a batch of rays (include/qsdvr_b200.h,
qsdvr_render_*).

* ``render_forward`` / ``render_backward`` / ``render_train`` call the C ABI directly;
* ``FusedRender`` is the ``autograd.Function`` whose backward recomputes every sample
  (memory O(rays): nothing per-sample is saved between forward and backward);
* ``DenseRenderGrid`` is a RenderGrid (models/render.py:209-237) whose SDF is a dense
  quadric grid [R^3][8] instead of separable layers, rendered by the fused kernels.

Ray batches are the reference's per-ray tables: ``rays`` int32 [N,4] (RayInfo),
``origin`` and ``dir`` float32 [N,3] (RayCut output after masking).
"""
from __future__ import annotations

import ctypes
import math

import torch
from torch import autograd, nn

from . import _lib
from ._lib import F32, I32, P, U32, call

STORAGE = {"f32": 0, "bf16": 1}
TRANSMITTANCE = {"product": 0, "log": 1}
MODES = {"compat": _lib.MODE_COMPAT, "fixed": _lib.MODE_FIXED}


class RenderArgs(ctypes.Structure):
    """qsdvr_render_args (include/qsdvr_b200.h)."""
    _fields_ = [("rays", P), ("origin", P), ("dir", P), ("ray_count", U32), ("reso", U32), ("interval", F32),
                ("logistic_coef", F32), ("mode", I32), ("storage", I32), ("transmittance", I32), ("sh_degree", I32),
                ("sdf_grid", P), ("data", P), ("color", P), ("target", P), ("grad_color", P), ("sdf_grad", P),
                ("data_grad", P), ("loss", P), ("grad_scale", F32), ("workspace", P), ("workspace_bytes", ctypes.c_uint64),
                ("sdf_layers", P), ("sdf_layers_grad", P), ("tlist", P), ("sample_alpha", P),
                ("sample_capacity", ctypes.c_uint64), ("order", P), ("data_grad_storage", I32),
                ("merge_scatter", I32)]


_lib.extra_signatures({
    "qsdvr_render_forward": [ctypes.POINTER(RenderArgs), P],
    "qsdvr_render_backward": [ctypes.POINTER(RenderArgs), P],
    "qsdvr_render_train": [ctypes.POINTER(RenderArgs), P],
    "qsdvr_separable_sdf_tables": [P, P, P, P, U32, P, P],
    "qsdvr_separable_sdf_grad": [P, U32, P, P, P, P, P],
    "qsdvr_ray_order_keys": [P, P, P, U32, F32, P, P],
    "qsdvr_sdf_cells_bf16": [P, P, ctypes.c_uint64, P],
    "qsdvr_ray_order": [P, P, P, U32, F32, P, P, ctypes.c_size_t, P],
    "qsdvr_ray_order_list": [P, P, P, U32, P, P, P, ctypes.c_size_t, P],
    "qsdvr_render_forward_bricks": [ctypes.POINTER(RenderArgs), P],
}, {"qsdvr_render_workspace_size": [ctypes.POINTER(RenderArgs)], "qsdvr_ray_order_workspace_size": [U32]})

_workspaces: dict = {}


def workspace(device, args: "RenderArgs") -> torch.Tensor:
    """A cached workspace for the persistent kernels on ``device`` (one per device and
    kernel configuration; launches on one stream never overlap, so it can be reused)."""
    key = (device, args.mode, args.storage, args.transmittance, args.sh_degree)
    need = int(_lib.lib().qsdvr_render_workspace_size(ctypes.byref(args)))
    ws = _workspaces.get(key)
    if ws is None or ws.numel() < need:
        ws = torch.empty(need, dtype=torch.uint8, device=device)
        _workspaces[key] = ws
    return ws


def _ptr(t):
    return t.data_ptr() if t is not None and t.numel() else None


def _check_batch(rays, origin, direction):
    dev = rays.device
    if not rays.is_cuda or rays.dtype != torch.int32 or rays.dim() != 2 or rays.shape[1] != 4:
        raise ValueError("rays must be a CUDA int32 [N,4] tensor")
    n = rays.shape[0]
    for t, nm in ((origin, "origin"), (direction, "dir")):
        if t.device != dev or t.dtype != torch.float32 or t.numel() != 3 * n or not t.is_contiguous():
            raise ValueError(f"{nm} must be a contiguous float32 [N,3] tensor on {dev}")
    if not rays.is_contiguous():
        raise ValueError("rays must be contiguous")
    return dev, n


def sh_degree_of(data, R) -> int:
    """SH degree implied by the appearance grid: 32-channel rows are degree 2 (the
    reference), 64-channel rows degree 3."""
    c = data.numel() // (R + 1) ** 3
    if c * (R + 1) ** 3 != data.numel() or c not in (32, 64):
        raise ValueError(f"data must be [(R+1)^3, 32] or [(R+1)^3, 64] for R={R}")
    return 2 if c == 32 else 3


def _grid_storage(sdf_grid, data, R):
    if sdf_grid.dtype != data.dtype or sdf_grid.dtype not in (torch.float32, torch.bfloat16):
        raise TypeError("sdf_grid and data must both be float32 or both bfloat16")
    if sdf_grid.numel() != 8 * R ** 3:
        raise ValueError(f"sdf_grid must be [R^3,8] for R={R}")
    sh_degree_of(data, R)
    if not (sdf_grid.is_contiguous() and data.is_contiguous()):
        raise ValueError("grids must be contiguous")
    return STORAGE["bf16" if sdf_grid.dtype == torch.bfloat16 else "f32"]


def make_args(rays, origin, direction, sdf_grid, data, reso, interval, k, mode="compat", transmittance="product",
              color=None, target=None, grad_color=None, sdf_grad=None, data_grad=None, loss=None,
              grad_scale=0.0, persistent=True, tlist=None, sample_alpha=None, sdf_layers=None,
              sdf_layers_grad=None, order=None, merge=False) -> RenderArgs:
    dev, n = _check_batch(rays, origin, direction)
    a = RenderArgs()
    a.rays, a.origin, a.dir = _ptr(rays), _ptr(origin), _ptr(direction)
    a.ray_count, a.reso = n, int(reso)
    a.interval, a.logistic_coef = float(interval), float(k)
    a.mode = MODES[mode]
    if sdf_layers is not None:
        rows = 3 * int(reso) + 1
        for t, nm in ((sdf_layers, "sdf_layers"), (sdf_layers_grad, "sdf_layers_grad")):
            if t is not None and (t.device != dev or t.dtype != torch.float32 or t.shape != (rows, 4)
                                  or not t.is_contiguous()):
                raise ValueError(f"{nm} must be a contiguous float32 [{rows},4] tensor on {dev}")
        if data.dtype not in (torch.float32, torch.bfloat16) or not data.is_contiguous():
            raise TypeError("data must be a contiguous float32 or bfloat16 tensor")
        sh_degree_of(data, int(reso))
        a.storage = STORAGE["bf16" if data.dtype == torch.bfloat16 else "f32"]
        a.sdf_layers, a.sdf_layers_grad = _ptr(sdf_layers), _ptr(sdf_layers_grad)
    else:
        a.storage = _grid_storage(sdf_grid, data, int(reso))
    a.transmittance = TRANSMITTANCE[transmittance]
    a.sh_degree = sh_degree_of(data, int(reso))
    a.sdf_grid, a.data = _ptr(sdf_grid), _ptr(data)
    a.color, a.target, a.grad_color = _ptr(color), _ptr(target), _ptr(grad_color)
    a.sdf_grad, a.data_grad, a.loss = _ptr(sdf_grad), _ptr(data_grad), _ptr(loss)
    a.grad_scale = float(grad_scale)
    a.merge_scatter = 1 if merge else 0
    a.workspace, a.workspace_bytes = None, 0
    if tlist is not None:
        _check_tlist(tlist, n, dev)
        a.tlist = tlist.data_ptr()
    if sample_alpha is not None:
        if sample_alpha.device != dev or sample_alpha.dtype != torch.float32 or not sample_alpha.is_contiguous():
            raise ValueError(f"sample_alpha must be a contiguous float32 tensor on {dev}")
        a.sample_alpha, a.sample_capacity = _ptr(sample_alpha), sample_alpha.numel()
    if data_grad is not None:
        if (data_grad.device != dev or data_grad.dtype not in (torch.float32, torch.bfloat16)
                or data_grad.numel() != data.numel() or not data_grad.is_contiguous()):
            raise ValueError("data_grad must be a contiguous float32 or bfloat16 tensor shaped like data")
        a.data_grad_storage = STORAGE["bf16" if data_grad.dtype == torch.bfloat16 else "f32"]
    if order is not None:
        if order.device != dev or order.dtype != torch.int32 or order.shape != (n,) or not order.is_contiguous():
            raise ValueError(f"order must be a contiguous int32 [N] permutation on {dev}")
        a.order = order.data_ptr()
    if persistent and n:
        with torch.cuda.device(dev):
            ws = workspace(dev, a)
        a.workspace, a.workspace_bytes = ws.data_ptr(), ws.numel()
    return a


def _stream(dev):
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def _check_tlist(tlist, n, dev):
    if tlist.device != dev or tlist.dtype != torch.float32 or tlist.shape != (n, 33) or not tlist.is_contiguous():
        raise ValueError(f"tlist must be a contiguous float32 [N,33] tensor on {dev}")


def ray_order(rays, origin, direction, interval, tlist=None) -> torch.Tensor:
    """A permutation (int32 [N]) that lists the rays by the Morton code of their in-box
    midpoint on a 32^3 lattice (qsdvr_ray_order: the library's counting sort), rays without
    samples last.  Passed as ``order`` to the render calls, neighbouring rays in the kernel's
    schedule cross neighbouring cells, so more of the gathered rows and gradient lines are found
    in L2.  With ``tlist`` (the [N,33] sample list of a list-mode render) each ray is keyed on
    its median SDF position instead (qsdvr_ray_order_list), so rays that hit the same patch of
    the surface run side by side."""
    dev, n = _check_batch(rays, origin, direction)
    if tlist is not None:
        _check_tlist(tlist, n, dev)
    order = torch.empty(n, dtype=torch.int32, device=dev)
    if n == 0:
        return order
    need = int(_lib.lib().qsdvr_ray_order_workspace_size(n))
    key = (dev, "order")
    ws = _workspaces.get(key)
    if ws is None or ws.numel() < need:
        ws = torch.empty(need, dtype=torch.uint8, device=dev)
        _workspaces[key] = ws
    with torch.cuda.device(dev):
        if tlist is None:
            call("qsdvr_ray_order", _ptr(rays), _ptr(origin), _ptr(direction), n, float(interval), _ptr(order),
                 ws.data_ptr(), ws.numel(), _stream(dev))
        else:
            call("qsdvr_ray_order_list", _ptr(rays), _ptr(origin), _ptr(direction), n, _ptr(tlist), _ptr(order),
                 ws.data_ptr(), ws.numel(), _stream(dev))
    return order


def ray_order_keys(rays, origin, direction, interval) -> torch.Tensor:
    """The 30-bit Morton codes of the rays' midpoints (qsdvr_ray_order_keys), int32 [N]."""
    dev, n = _check_batch(rays, origin, direction)
    keys = torch.empty(n, dtype=torch.int32, device=dev)
    with torch.cuda.device(dev):
        call("qsdvr_ray_order_keys", _ptr(rays), _ptr(origin), _ptr(direction), n, float(interval), _ptr(keys),
             _stream(dev))
    return keys


def render_forward(rays, origin, direction, sdf_grid, data, reso, interval, k, mode="compat",
                   transmittance="product", color=None, persistent=True, tlist=None, sample_alpha=None,
                   sdf_layers=None, order=None):
    """Colour of every ray [N,3].  ``tlist`` [N,33]: render at those SDF positions (32 render
    samples per ray at their midpoints) instead of the uniform march; ``sample_alpha``: also
    write every render sample's alpha at the ray's render offset; ``sdf_layers`` (with
    ``sdf_grid`` None): the separable SDF tables of ``separable_tables``; ``order``: the
    order in which the kernel takes the rays (``ray_order``)."""
    dev, n = _check_batch(rays, origin, direction)
    if color is None:
        color = torch.empty((n, 3), dtype=torch.float32, device=dev)
    a = make_args(rays, origin, direction, sdf_grid, data, reso, interval, k, mode, transmittance, color=color,
                  persistent=persistent, tlist=tlist, sample_alpha=sample_alpha, sdf_layers=sdf_layers, order=order)
    with torch.cuda.device(dev):
        call("qsdvr_render_forward", ctypes.byref(a), _stream(dev))
    return color


def render_forward_bricks(rays, origin, direction, sdf_grid, data, reso, interval, k, color=None):
    """Colour of every ray [N,3] by the brick-staged frame forward (qsdvr_render_forward_bricks:
    fixed mode, uniform march, log transmittance; 128-byte vertex rows, i.e. bf16 SH degree 3
    or fp32 degree 2).  Meant for a frame's rays listed tile by tile (8 x 8 pixels,
    ``Camera.GenerateRayPoints(order="tiles")``): each block of 64 rays shares one staged brick
    of the appearance grid per round."""
    dev, n = _check_batch(rays, origin, direction)
    if color is None:
        color = torch.empty((n, 3), dtype=torch.float32, device=dev)
    a = make_args(rays, origin, direction, sdf_grid, data, reso, interval, k, "fixed", "log", color=color,
                  persistent=False)
    with torch.cuda.device(dev):
        call("qsdvr_render_forward_bricks", ctypes.byref(a), _stream(dev))
    return color


def render_backward(grad_color, rays, origin, direction, sdf_grid, data, reso, interval, k, sdf_grad, data_grad,
                    mode="compat", transmittance="product", persistent=True, tlist=None, sdf_layers=None,
                    order=None, merge=False):
    """Accumulate dL/d(sdf_grid) (fp32) and dL/d(data) (fp32, or bf16 when ``data_grad`` is a
    bfloat16 tensor) for a given dL/dcolor.  With ``sdf_layers``, ``sdf_grad`` is the tables'
    gradient ([3R+1,4], see ``separable_grad``)."""
    dev, n = _check_batch(rays, origin, direction)
    sdf_src = sdf_layers if sdf_layers is not None else sdf_grid
    if (sdf_grad.dtype != torch.float32 or sdf_grad.numel() != sdf_src.numel() or sdf_grad.device != dev
            or not sdf_grad.is_contiguous()):
        raise ValueError("sdf_grad must be a contiguous float32 tensor shaped like its grid")
    g = grad_color.contiguous().float()
    a = make_args(rays, origin, direction, sdf_grid, data, reso, interval, k, mode, transmittance, grad_color=g,
                  sdf_grad=None if sdf_layers is not None else sdf_grad, data_grad=data_grad,
                  persistent=persistent, tlist=tlist, sdf_layers=sdf_layers,
                  sdf_layers_grad=sdf_grad if sdf_layers is not None else None, order=order, merge=merge)
    with torch.cuda.device(dev):
        call("qsdvr_render_backward", ctypes.byref(a), _stream(dev))


def render_train(target, rays, origin, direction, sdf_grid, data, reso, interval, k, sdf_grad, data_grad,
                 mode="compat", transmittance="product", loss=None, color=None, persistent=True, tlist=None,
                 sample_alpha=None, sdf_layers=None, order=None, merge=False):
    """Forward + MSE (mean over N x 3) + backward in one launch.  Returns (color, loss_sum)
    where loss_sum accumulates sum |color - target|^2 (divide by 3N for the mean).  With
    ``sdf_layers``, ``sdf_grad`` is the tables' gradient ([3R+1,4]).  A bfloat16 ``data_grad``
    accumulates the appearance gradient in bf16 (half its traffic; the SDF gradient stays
    fp32).  ``merge``: samples of a warp chunk in the same cell send one summed appearance
    RED per corner row (the kernel's same-cell merge)."""
    dev, n = _check_batch(rays, origin, direction)
    if color is None:
        color = torch.empty((n, 3), dtype=torch.float32, device=dev)
    if loss is None:
        loss = torch.zeros(1, dtype=torch.float32, device=dev)
    sep = sdf_layers is not None
    a = make_args(rays, origin, direction, sdf_grid, data, reso, interval, k, mode, transmittance, color=color,
                  target=target.contiguous(), sdf_grad=None if sep else sdf_grad, data_grad=data_grad, loss=loss,
                  grad_scale=2.0 / (3.0 * max(n, 1)), persistent=persistent, tlist=tlist,
                  sample_alpha=sample_alpha, sdf_layers=sdf_layers, sdf_layers_grad=sdf_grad if sep else None,
                  order=order, merge=merge)
    with torch.cuda.device(dev):
        call("qsdvr_render_train", ctypes.byref(a), _stream(dev))
    return color, loss


class FusedRender(autograd.Function):
    """Differentiable fused render.  Forward saves only its inputs; backward recomputes
    each sample's alpha, transmittance and colour (memory O(rays))."""

    @staticmethod
    def forward(ctx, sdf_grid, data, rays, origin, direction, reso, interval, k, mode, transmittance):
        color = render_forward(rays, origin, direction, sdf_grid.detach(), data.detach(), reso, interval, k, mode,
                               transmittance)
        ctx.save_for_backward(sdf_grid, data, rays, origin, direction)
        ctx.cfg = (reso, interval, k, mode, transmittance)
        return color

    @staticmethod
    def backward(ctx, grad_color):
        sdf_grid, data, rays, origin, direction = ctx.saved_tensors
        reso, interval, k, mode, transmittance = ctx.cfg
        sg = torch.zeros(sdf_grid.shape, dtype=torch.float32, device=sdf_grid.device)
        dg = torch.zeros(data.shape, dtype=torch.float32, device=data.device)
        render_backward(grad_color, rays, origin, direction, sdf_grid.detach(), data.detach(), reso, interval, k, sg,
                        dg, mode, transmittance)
        return sg.to(sdf_grid.dtype), dg.to(data.dtype), None, None, None, None, None, None, None, None


def sdf_cells_bf16(grid8: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """BF16 storage copy [R^3,8] of an fp32 quadric cell grid (qsdvr_sdf_cells_bf16): a0..a5
    rounded to nearest, a6 rescaled so the stored cell's SDF at its centre equals the
    master's, held as two bf16 (slots 6 and 7) that the kernels add."""
    if not grid8.is_cuda or grid8.dtype != torch.float32 or grid8.dim() != 2 or grid8.shape[1] != 8 \
            or not grid8.is_contiguous():
        raise ValueError("grid8 must be a contiguous CUDA float32 [cells, 8] tensor")
    if out is None:
        out = torch.empty(grid8.shape, dtype=torch.bfloat16, device=grid8.device)
    elif out.dtype != torch.bfloat16 or out.shape != grid8.shape or out.device != grid8.device \
            or not out.is_contiguous():
        raise ValueError("out must be a contiguous bfloat16 tensor shaped like grid8")
    with torch.cuda.device(grid8.device):
        call("qsdvr_sdf_cells_bf16", _ptr(grid8), _ptr(out), grid8.shape[0], _stream(grid8.device))
    return out


def pad_grid7(grid7: torch.Tensor) -> torch.Tensor:
    """[R^3,7] (reference layout) -> [R^3,8] (16-byte-aligned rows, a7 = 0)."""
    g = grid7.reshape(-1, 7)
    out = torch.zeros((g.shape[0], 8), dtype=g.dtype, device=g.device)
    out[:, :7] = g
    return out


class DenseRenderGrid(nn.Module):
    """RenderGrid with a dense quadric SDF grid, rendered by the fused kernels.

    Parameters are fp32 masters; with ``storage='bf16'`` the kernels read bf16 copies
    refreshed by ``sync_storage()`` (call it after each optimizer step)."""

    def __init__(self, reso: int = 128, logisticCoef: float = 5.0, interval: float = 4.0 / 256, mode: str = "compat",
                 storage: str = "f32", transmittance: str | None = None, device="cuda", sdf_grid=None, data=None,
                 sh_degree: int = 2):
        super().__init__()
        self.reso, self.interval, self.mode, self.storage = reso, interval, mode, storage
        self.logisticCoef = logisticCoef
        self.transmittance = transmittance or ("log" if storage == "bf16" else "product")
        if sdf_grid is None:
            from .scenes import sphere_grid

            sdf_grid = sphere_grid(reso, 0.5, 0.0, device=device)
        if data is None:
            # models/render.py:215-223 (ao 1, metallic 0.1, diffuse 1, SH DC 0.5); degree 3
            # keeps the same values after its 48 SH channels
            nsh = 3 * (sh_degree + 1) ** 2
            data = torch.zeros(((reso + 1) ** 3, 32 if sh_degree == 2 else 64), dtype=torch.float32, device=device)
            data[:, nsh + 4] = 1
            data[:, nsh + 3] = 0.1
            data[:, nsh:nsh + 3] = 1
            data[:, 0:3] = 0.5
        g = sdf_grid.reshape(-1, sdf_grid.shape[-1])
        self.sdfGrid = nn.Parameter(pad_grid7(g) if g.shape[1] == 7 else g.contiguous().clone())
        self.renderData = nn.Parameter(data.reshape((reso + 1) ** 3, -1).contiguous().clone())
        self._copies = None
        self.sync_storage()

    def sync_storage(self):
        """Refresh the bf16 copies from the fp32 masters (in place once they exist, so tensors
        handed out earlier stay valid).  A model held on the CPU is never rendered (the kernels
        run on CUDA devices only); its SDF copy is the plain bf16 rounding, which the kernels
        read the same way, until the model is synced on a GPU."""
        if self.storage != "bf16":
            return
        sdf, data = self.sdfGrid.detach(), self.renderData.detach()
        if self._copies is None:
            self._copies = (torch.empty(sdf.shape, dtype=torch.bfloat16, device=sdf.device),
                            torch.empty(data.shape, dtype=torch.bfloat16, device=data.device))
        if sdf.is_cuda:
            sdf_cells_bf16(sdf, out=self._copies[0])
        else:
            self._copies[0].copy_(sdf)
        self._copies[1].copy_(data)

    def grids(self):
        if self.storage == "bf16":
            return self._copies
        return self.sdfGrid, self.renderData

    def forward(self, rays, origin, direction):
        if self.storage == "bf16":
            return _Bf16Render.apply(self.sdfGrid, self.renderData, self._copies[0], self._copies[1], rays, origin,
                                     direction, self)
        return FusedRender.apply(self.sdfGrid, self.renderData, rays, origin, direction, self.reso, self.interval,
                                 self.logisticCoef, self.mode, self.transmittance)

    def set_logisticCoef(self, logisticCoef):
        self.logisticCoef = logisticCoef


class _Bf16Render(autograd.Function):
    """Forward/backward on the bf16 copies; gradients (fp32) flow to the fp32 masters."""

    @staticmethod
    def forward(ctx, sdf_master, data_master, sdf_bf16, data_bf16, rays, origin, direction, model):
        ctx.save_for_backward(sdf_bf16, data_bf16, rays, origin, direction)
        ctx.model = model
        return render_forward(rays, origin, direction, sdf_bf16, data_bf16, model.reso, model.interval,
                              model.logisticCoef, model.mode, model.transmittance)

    @staticmethod
    def backward(ctx, grad_color):
        sdf_bf16, data_bf16, rays, origin, direction = ctx.saved_tensors
        m = ctx.model
        sg = torch.zeros(sdf_bf16.shape, dtype=torch.float32, device=sdf_bf16.device)
        dg = torch.zeros(data_bf16.shape, dtype=torch.float32, device=data_bf16.device)
        render_backward(grad_color, rays, origin, direction, sdf_bf16, data_bf16, m.reso, m.interval, m.logisticCoef,
                        sg, dg, m.mode, m.transmittance)
        return sg, dg, None, None, None, None, None, None


# ----------------------------------------------------------------------------- separable SDF

def separable_tables(x_layer, y_layer, z_layer, offset) -> torch.Tensor:
    """[3R+1, 4] tables of the separable quadric grid (models/render.py:172-207 layers +
    offset; the per-axis recurrences of LayerToGridForward, kernel/surface.cu:161-178)."""
    R = x_layer.numel()
    dev = x_layer.device
    for t, nm, nn_ in ((x_layer, "x_layer", R), (y_layer, "y_layer", R), (z_layer, "z_layer", R), (offset, "offset", 4)):
        if not t.is_cuda or t.device != dev or t.dtype != torch.float32 or t.numel() != nn_ or not t.is_contiguous():
            raise ValueError(f"{nm} must be a contiguous float32 CUDA tensor of {nn_} values on {dev}")
    out = torch.empty((3 * R + 1, 4), dtype=torch.float32, device=dev)
    with torch.cuda.device(dev):
        call("qsdvr_separable_sdf_tables", _ptr(x_layer), _ptr(y_layer), _ptr(z_layer), _ptr(offset), R, _ptr(out),
             _stream(dev))
    return out


def separable_grad(table_grad: torch.Tensor):
    """(x, y, z layer gradients [R], offset gradient [4]) from the tables' gradient, which
    the call consumes (the reverse recurrences run in place)."""
    R = (table_grad.shape[0] - 1) // 3
    dev = table_grad.device
    if table_grad.dtype != torch.float32 or table_grad.shape != (3 * R + 1, 4) or not table_grad.is_contiguous():
        raise ValueError("table_grad must be a contiguous float32 [3R+1,4] tensor")
    xg, yg, zg = (torch.empty(R, dtype=torch.float32, device=dev) for _ in range(3))
    og = torch.empty(4, dtype=torch.float32, device=dev)
    with torch.cuda.device(dev):
        call("qsdvr_separable_sdf_grad", _ptr(table_grad), R, _ptr(xg), _ptr(yg), _ptr(zg), _ptr(og), _stream(dev))
    return xg, yg, zg, og


class _SeparableRender(autograd.Function):
    @staticmethod
    def forward(ctx, x_layer, y_layer, z_layer, offset, data, rays, origin, direction, cfg):
        reso, interval, k, mode, transmittance = cfg
        tables = separable_tables(x_layer.detach(), y_layer.detach(), z_layer.detach(), offset.detach())
        color = render_forward(rays, origin, direction, None, data.detach(), reso, interval, k, mode, transmittance,
                               sdf_layers=tables)
        ctx.save_for_backward(tables, data, rays, origin, direction)
        ctx.cfg = cfg
        return color

    @staticmethod
    def backward(ctx, grad_color):
        tables, data, rays, origin, direction = ctx.saved_tensors
        reso, interval, k, mode, transmittance = ctx.cfg
        tg = torch.zeros_like(tables)
        dg = torch.zeros(data.shape, dtype=torch.float32, device=data.device)
        render_backward(grad_color, rays, origin, direction, None, data.detach(), reso, interval, k, tg, dg, mode,
                        transmittance, sdf_layers=tables)
        xg, yg, zg, og = separable_grad(tg)
        return xg, yg, zg, og, dg.to(data.dtype), None, None, None, None


class SeparableRenderGrid(nn.Module):
    """The reference RenderGrid (models/render.py:172-237: QuadricGrid layers + offset and the
    [(R+1)^3,32] appearance grid, same initial values) rendered and differentiated by the fused
    kernels.  The [R^3,7] cell grid is never materialised: the kernels assemble each cell from
    O(R) per-axis tables and reduce its gradient back into them."""

    def __init__(self, reso: int = 128, logisticCoef: float = 5.0, interval: float = 4.0 / 256, mode: str = "compat",
                 transmittance: str = "product", device="cuda"):
        super().__init__()
        self.reso, self.interval, self.mode, self.transmittance = reso, interval, mode, transmittance
        self.logisticCoef = logisticCoef
        dev = torch.device(device)
        self.xLayer = nn.Parameter(torch.ones(reso, dtype=torch.float32, device=dev))
        self.yLayer = nn.Parameter(torch.ones(reso, dtype=torch.float32, device=dev))
        self.zLayer = nn.Parameter(torch.ones(reso, dtype=torch.float32, device=dev))
        c = -reso  # models/render.py:187-192
        self.offset = nn.Parameter(torch.tensor([-2.0 * c, -2.0 * c, -2.0 * c, math.sqrt(3 * c * c)],
                                                dtype=torch.float32, device=dev))
        data = torch.zeros(((reso + 1) ** 3, 32), dtype=torch.float32, device=dev)
        data[:, 31] = 1  # models/render.py:215-223
        data[:, 30] = 0.1
        data[:, 27:30] = 1
        data[:, 0:3] = 0.5
        self.renderData = nn.Parameter(data)

    def cfg(self):
        return (self.reso, self.interval, self.logisticCoef, self.mode, self.transmittance)

    def forward(self, rays, origin, direction):
        return _SeparableRender.apply(self.xLayer, self.yLayer, self.zLayer, self.offset, self.renderData, rays, origin,
                                      direction, self.cfg())

    def train_step(self, target, rays, origin, direction, loss=None):
        """Forward + MSE + backward in one fused launch; accumulates into the parameters' .grad.
        Returns (colour, loss_sum)."""
        tables = separable_tables(self.xLayer.detach(), self.yLayer.detach(), self.zLayer.detach(),
                                  self.offset.detach())
        tg = torch.zeros_like(tables)
        if self.renderData.grad is None:
            self.renderData.grad = torch.zeros_like(self.renderData)
        color, loss = render_train(target, rays, origin, direction, None, self.renderData.detach(), self.reso,
                                   self.interval, self.logisticCoef, tg, self.renderData.grad, self.mode,
                                   self.transmittance, loss=loss, sdf_layers=tables)
        for p, g in zip((self.xLayer, self.yLayer, self.zLayer, self.offset), separable_grad(tg)):
            p.grad = g if p.grad is None else p.grad.add_(g)
        return color, loss

    def set_logisticCoef(self, logisticCoef):
        self.logisticCoef = logisticCoef
