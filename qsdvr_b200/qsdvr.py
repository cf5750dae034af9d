"""Drop-in replacement of the reference's ``qsdvr`` extension module (kernel/qsdvr.cpp:5-50).

Same 14 function names, argument order, in-place output convention and pre-zeroed
gradient contract as the reference, plus the ``CameraArgs`` class.  Each function
validates its tensors (device, dtype, contiguity, shapes) and raises instead of
misbehaving silently, then calls the C ABI (include/qsdvr_b200.h) on torch's current
CUDA stream.  ``import qsdvr_b200.qsdvr as qsdvr`` is all a caller of the reference needs.

Differences in behaviour from the reference, all deliberate:
  * errors raise (the reference has no checks at all);
  * RayCut scans on the device and synchronises only to read the two totals;
  * LayerToGridBackward writes exactly 4 floats of ``offset`` (the reference copies
    R floats into it, overrunning the 4-float tensor).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import call

__all__ = ["CameraArgs", "GridInterpolationForward", "GridInterpolationBackward", "LayerToGridForward",
           "LayerToGridBackward", "SampleSDFForward", "SampleSDFBackward", "SampleNormalForward",
           "SampleNormalBackward", "ShaderForward", "ShaderBackward", "RayAggregateForward",
           "RayAggregateBackward", "RayCut", "GenerateRayPoints"]

_MODES = {"compat": _lib.MODE_COMPAT, "fixed": _lib.MODE_FIXED}


class CameraArgs:
    """kernel/qsdvr.cpp:36-50 / include/camera.h:19-34 (PyCameraArgs).

    ``rotation`` (row-major 3x3 camera-to-world) and ``translation`` are float32 arrays;
    ``pixelCount`` is set by the caller, ``sdfCount``/``renderCount`` by RayCut.
    """

    def __init__(self):
        self.width = 0
        self.height = 0
        self._rotation = np.zeros(9, np.float32)
        self._translation = np.zeros(3, np.float32)
        self.fx = self.fy = self.cx = self.cy = 0.0
        self.near = self.far = 0.0
        self.pixelCount = 0
        self.sdfCount = 0
        self.renderCount = 0

    @property
    def rotation(self):
        return self._rotation

    @rotation.setter
    def rotation(self, v):
        self._rotation = np.ascontiguousarray(np.asarray(v, dtype=np.float32).reshape(-1))

    @property
    def translation(self):
        return self._translation

    @translation.setter
    def translation(self, v):
        self._translation = np.ascontiguousarray(np.asarray(v, dtype=np.float32).reshape(-1))

    def to_c(self) -> _lib.Camera:
        if self._rotation.size != 9 or self._translation.size != 3:
            raise ValueError("CameraArgs: rotation needs 9 and translation 3 values")
        c = _lib.Camera()
        c.width, c.height = int(self.width), int(self.height)
        for i in range(9):
            c.rotation[i] = float(self._rotation[i])
        for i in range(3):
            c.translation[i] = float(self._translation[i])
        c.fx, c.fy, c.cx, c.cy = float(self.fx), float(self.fy), float(self.cx), float(self.cy)
        c.near_depth, c.far_depth = float(self.near), float(self.far)
        return c


# ----------------------------------------------------------------------------- validation

def _check(t, name, dtype, device=None, shape=None, cuda=True):
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name}: expected a torch.Tensor, got {type(t).__name__}")
    if t.dtype != dtype:
        raise TypeError(f"{name}: expected dtype {dtype}, got {t.dtype}")
    if cuda and not t.is_cuda:
        raise ValueError(f"{name}: expected a CUDA tensor")
    if device is not None and t.device != device:
        raise ValueError(f"{name}: expected device {device}, got {t.device}")
    if not t.is_contiguous():
        raise ValueError(f"{name}: expected a contiguous tensor")
    if shape is not None:
        if t.dim() != len(shape) or any(s is not None and a != s for a, s in zip(t.shape, shape)):
            raise ValueError(f"{name}: expected shape {tuple(shape)}, got {tuple(t.shape)}")
    return t


def _p(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr() if t is not None and t.numel() else 0)


def _stream(device) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _rows(t, name, width, device, dtype=torch.float32):
    _check(t, name, dtype, device)
    if t.numel() % width:
        raise ValueError(f"{name}: size {t.numel()} is not a multiple of {width}")
    return t.numel() // width


# ----------------------------------------------------------------------------- render.cu

def GridInterpolationForward(dataGrid, pointList, indexList, out, reso):
    """kernel/render.cu:317-323: out[i] = trilinear fetch of dataGrid at sample i."""
    dev = _check(dataGrid, "dataGrid", torch.float32).device
    n = _rows(pointList, "pointList", 3, dev)
    _check(indexList, "indexList", torch.int32, dev, (n,))
    _check(out, "out", torch.float32, dev)
    if dataGrid.shape[-1] != 32 or out.numel() != 32 * n:
        raise ValueError("GridInterpolationForward: 32 channels per vertex and out of [N,32] expected")
    with torch.cuda.device(dev):
        call("qsdvr_grid_interpolation_forward", _p(dataGrid), _p(pointList), _p(indexList), _p(out), n, int(reso),
             dataGrid.numel() // 32, _stream(dev))


def GridInterpolationBackward(dataGrid, pointList, indexList, out, reso):
    """kernel/render.cu:325-331: accumulate the adjoint of out into dataGrid (pre-zeroed)."""
    dev = _check(dataGrid, "dataGrid", torch.float32).device
    n = _rows(pointList, "pointList", 3, dev)
    _check(indexList, "indexList", torch.int32, dev, (n,))
    _check(out, "out", torch.float32, dev)
    if dataGrid.shape[-1] != 32 or out.numel() != 32 * n:
        raise ValueError("GridInterpolationBackward: 32 channels per vertex and gradient of [N,32] expected")
    with torch.cuda.device(dev):
        call("qsdvr_grid_interpolation_backward", _p(dataGrid), _p(pointList), _p(indexList), _p(out), n, int(reso),
             dataGrid.numel() // 32, _stream(dev))


def ShaderForward(out, normalList, viewDirList, dataList, specularList, *, mode="compat"):
    """kernel/render.cu:333-339.  ``mode='compat'`` reproduces the reference's SH read."""
    dev = _check(dataList, "dataList", torch.float32).device
    n = _rows(normalList, "normalList", 3, dev)
    for t, nm in ((viewDirList, "viewDirList"), (out, "out"), (specularList, "specularList")):
        if _rows(t, nm, 3, dev) != n:
            raise ValueError(f"ShaderForward: {nm} has {t.numel() // 3} rows, expected {n}")
    if _rows(dataList, "dataList", 32, dev) != n:
        raise ValueError("ShaderForward: dataList must be [N,32]")
    with torch.cuda.device(dev):
        call("qsdvr_shader_forward", _p(out), _p(normalList), _p(viewDirList), _p(dataList), _p(specularList), n,
             _MODES[mode], _stream(dev))


def ShaderBackward(out, normalList, viewDirList, dataList, specularList, normalGradList, dataGradList, *,
                   mode="compat"):
    """kernel/render.cu:341-347.  ``out`` is the incoming gradient of the shaded colour."""
    dev = _check(dataList, "dataList", torch.float32).device
    n = _rows(normalList, "normalList", 3, dev)
    for t, nm in ((viewDirList, "viewDirList"), (out, "out"), (specularList, "specularList"),
                  (normalGradList, "normalGradList")):
        if _rows(t, nm, 3, dev) != n:
            raise ValueError(f"ShaderBackward: {nm} has {t.numel() // 3} rows, expected {n}")
    if _rows(dataList, "dataList", 32, dev) != n or _rows(dataGradList, "dataGradList", 32, dev) != n:
        raise ValueError("ShaderBackward: dataList/dataGradList must be [N,32]")
    with torch.cuda.device(dev):
        call("qsdvr_shader_backward", _p(out), _p(normalList), _p(viewDirList), _p(dataList), _p(specularList),
             _p(normalGradList), _p(dataGradList), n, _MODES[mode], _stream(dev))


def _rays(rayList, dev):
    _check(rayList, "rayList", torch.int32, dev)
    if rayList.dim() != 2 or rayList.shape[1] != 4:
        raise ValueError("rayList must be int32 [N,4] (sdfCount, sdfOffset, renderCount, renderOffset)")
    return rayList.shape[0]


def RayAggregateForward(out, rgbList, sdfList, rayList, alphaList, TList, logisticCoef):
    """kernel/render.cu:349-355: NeuS alpha + compositing; stores alpha and T per sample."""
    dev = _check(rgbList, "rgbList", torch.float32).device
    nr = _rays(rayList, dev)
    m = _rows(rgbList, "rgbList", 3, dev)
    s = _rows(sdfList, "sdfList", 1, dev)
    if _rows(out, "out", 3, dev) != nr or _rows(alphaList, "alphaList", 1, dev) < m or _rows(TList, "TList", 1, dev) < m:
        raise ValueError("RayAggregateForward: out must be [N,3], alphaList/TList as long as rgbList")
    with torch.cuda.device(dev):
        call("qsdvr_ray_aggregate_forward", _p(out), _p(rgbList), _p(sdfList), _p(rayList), _p(alphaList), _p(TList),
             nr, float(logisticCoef), s, m, _stream(dev))


def RayAggregateBackward(outgrad, rgbList, sdfList, rayList, alphaList, TList, rgbGradList, sdfGradList,
                         logisticCoef):
    """kernel/render.cu:357-363: writes rgbGradList and sdfGradList for every ray sample."""
    dev = _check(rgbList, "rgbList", torch.float32).device
    nr = _rays(rayList, dev)
    m = _rows(rgbList, "rgbList", 3, dev)
    s = _rows(sdfList, "sdfList", 1, dev)
    if (_rows(outgrad, "outgrad", 3, dev) != nr or _rows(rgbGradList, "rgbGradList", 3, dev) != m
            or _rows(sdfGradList, "sdfGradList", 1, dev) != s or _rows(alphaList, "alphaList", 1, dev) < m
            or _rows(TList, "TList", 1, dev) < m):
        raise ValueError("RayAggregateBackward: inconsistent shapes")
    with torch.cuda.device(dev):
        call("qsdvr_ray_aggregate_backward", _p(outgrad), _p(rgbList), _p(sdfList), _p(rayList), _p(alphaList),
             _p(TList), _p(rgbGradList), _p(sdfGradList), nr, float(logisticCoef), s, m, _stream(dev))


# ----------------------------------------------------------------------------- surface.cu

def _grid7(sdfGrid, name, dev=None):
    _check(sdfGrid, name, torch.float32, dev)
    if sdfGrid.numel() % 7:
        raise ValueError(f"{name}: expected [R,R,R,7]")
    return sdfGrid.numel() // 7


def SampleSDFForward(out, sdfGrid, pointList, indexList, reso):
    """kernel/surface.cu:343-350."""
    dev = sdfGrid.device
    cells = _grid7(sdfGrid, "sdfGrid")
    n = _rows(pointList, "pointList", 3, dev)
    _check(indexList, "indexList", torch.int32, dev, (n,))
    if _rows(out, "out", 1, dev) != n:
        raise ValueError("SampleSDFForward: out must have one value per point")
    with torch.cuda.device(dev):
        call("qsdvr_sample_sdf_forward", _p(out), _p(sdfGrid), _p(pointList), _p(indexList), n, float(reso), cells,
             _stream(dev))


def SampleSDFBackward(out, sdfGrid, pointList, indexList, sdfGradGrid, reso):
    """kernel/surface.cu:352-359 (accumulates into sdfGradGrid)."""
    dev = sdfGrid.device
    cells = _grid7(sdfGrid, "sdfGrid")
    if _grid7(sdfGradGrid, "sdfGradGrid", dev) != cells:
        raise ValueError("SampleSDFBackward: sdfGradGrid must match sdfGrid")
    n = _rows(pointList, "pointList", 3, dev)
    _check(indexList, "indexList", torch.int32, dev, (n,))
    if _rows(out, "out", 1, dev) != n:
        raise ValueError("SampleSDFBackward: gradient must have one value per point")
    with torch.cuda.device(dev):
        call("qsdvr_sample_sdf_backward", _p(out), _p(sdfGrid), _p(pointList), _p(indexList), _p(sdfGradGrid), n,
             float(reso), cells, _stream(dev))


def SampleNormalForward(out, sdfGrid, pointList, indexList):
    """kernel/surface.cu:361-367."""
    dev = sdfGrid.device
    cells = _grid7(sdfGrid, "sdfGrid")
    n = _rows(pointList, "pointList", 3, dev)
    _check(indexList, "indexList", torch.int32, dev, (n,))
    if _rows(out, "out", 3, dev) != n:
        raise ValueError("SampleNormalForward: out must be [N,3]")
    with torch.cuda.device(dev):
        call("qsdvr_sample_normal_forward", _p(out), _p(sdfGrid), _p(pointList), _p(indexList), n, cells,
             _stream(dev))


def SampleNormalBackward(out, sdfGrid, pointList, indexList, sdfGradGrid):
    """kernel/surface.cu:369-375 (accumulates into sdfGradGrid)."""
    dev = sdfGrid.device
    cells = _grid7(sdfGrid, "sdfGrid")
    if _grid7(sdfGradGrid, "sdfGradGrid", dev) != cells:
        raise ValueError("SampleNormalBackward: sdfGradGrid must match sdfGrid")
    n = _rows(pointList, "pointList", 3, dev)
    _check(indexList, "indexList", torch.int32, dev, (n,))
    if _rows(out, "out", 3, dev) != n:
        raise ValueError("SampleNormalBackward: gradient must be [N,3]")
    with torch.cuda.device(dev):
        call("qsdvr_sample_normal_backward", _p(out), _p(sdfGrid), _p(pointList), _p(indexList), _p(sdfGradGrid), n,
             cells, _stream(dev))


def LayerToGridForward(out, xLayer, yLayer, zLayer, offset):
    """kernel/surface.cu:148-229.  Layers/offset may live on the CPU (as in the reference)."""
    dev = _check(out, "out", torch.float32).device
    R = xLayer.numel()
    if out.numel() != R ** 3 * 7 or yLayer.numel() != R or zLayer.numel() != R or offset.numel() < 4:
        raise ValueError("LayerToGridForward: out [R,R,R,7], three layers [R] and offset [4] expected")
    for t, nm in ((xLayer, "xLayer"), (yLayer, "yLayer"), (zLayer, "zLayer"), (offset, "offset")):
        _check(t, nm, torch.float32, cuda=False)
    with torch.cuda.device(dev):
        x, y, z = (t.to(dev, non_blocking=True) for t in (xLayer, yLayer, zLayer))
        off = offset.reshape(-1)[:4].to(dev, non_blocking=True).contiguous()
        ws = torch.empty(_lib.size("qsdvr_layer_to_grid_workspace_size", R), dtype=torch.uint8, device=dev)
        call("qsdvr_layer_to_grid_forward", _p(out), _p(x), _p(y), _p(z), _p(off), R, _p(ws), ws.numel(),
             _stream(dev))


def LayerToGridBackward(out, xLayer, yLayer, zLayer, offset):
    """kernel/surface.cu:231-341.  ``out`` is the [R,R,R,7] gradient; the layer tensors and
    offset[0:4] receive the layer gradients (written, not accumulated)."""
    dev = _check(out, "out", torch.float32).device
    R = xLayer.numel()
    if out.numel() != R ** 3 * 7 or yLayer.numel() != R or zLayer.numel() != R or offset.numel() < 4:
        raise ValueError("LayerToGridBackward: gradient [R,R,R,7], three layers [R] and offset [4] expected")
    with torch.cuda.device(dev):
        g = torch.empty(3 * R + 4, dtype=torch.float32, device=dev)
        ws = torch.empty(_lib.size("qsdvr_layer_to_grid_workspace_size", R), dtype=torch.uint8, device=dev)
        call("qsdvr_layer_to_grid_backward", _p(out), R, _p(g[:R]), _p(g[R:2 * R]), _p(g[2 * R:3 * R]),
             _p(g[3 * R:]), _p(ws), ws.numel(), _stream(dev))
        xLayer.copy_(g[:R].view_as(xLayer))
        yLayer.copy_(g[R:2 * R].view_as(yLayer))
        zLayer.copy_(g[2 * R:3 * R].view_as(zLayer))
        offset.reshape(-1)[:4].copy_(g[3 * R:])


# ----------------------------------------------------------------------------- camera.cu

def RayCut(args: CameraArgs, mask, rayList, originList, dirList, interval):
    """kernel/camera.cu:98-130.  Sets args.sdfCount / args.renderCount."""
    dev = _check(rayList, "rayList", torch.int32).device
    P = int(args.pixelCount)
    if rayList.shape != (P, 4) and rayList.numel() != 4 * P:
        raise ValueError(f"RayCut: rayList must be [{P},4]")
    _check(originList, "originList", torch.float32, dev)
    _check(dirList, "dirList", torch.float32, dev)
    if originList.numel() < 3 * P or dirList.numel() < 3 * P or mask.numel() < P:
        raise ValueError("RayCut: originList/dirList need [pixelCount,3], mask [pixelCount]")
    cam = args.to_c()
    with torch.cuda.device(dev):
        m = mask.reshape(-1)[:P].to(dev, torch.uint8, non_blocking=True).contiguous()
        ws = torch.empty(_lib.size("qsdvr_ray_cut_workspace_size", P), dtype=torch.uint8, device=dev)
        totals = torch.empty(2, dtype=torch.int32, device=dev)
        call("qsdvr_ray_cut", ctypes.byref(cam), _p(m), _p(rayList), _p(originList), _p(dirList), float(interval), P,
             _p(totals), _p(ws), ws.numel(), _stream(dev))
        t = totals.cpu()
    args.sdfCount = int(t[0])
    args.renderCount = int(t[1])


def GenerateRayPoints(args, sdfPointList, sdfIndexList, renderPointList, renderIndexList, viewDirList, rayList,
                      originList, dirList, interval, baseVolumeReso):
    """kernel/camera.cu:132-147."""
    dev = _check(rayList, "rayList", torch.int32).device
    n = _rays(rayList, dev)
    if _rows(originList, "originList", 3, dev) < n or _rows(dirList, "dirList", 3, dev) < n:
        raise ValueError("GenerateRayPoints: originList/dirList need one row per ray")
    s = _rows(sdfPointList, "sdfPointList", 3, dev)
    _check(sdfIndexList, "sdfIndexList", torch.int32, dev, (s,))
    m = _rows(renderPointList, "renderPointList", 3, dev)
    _check(renderIndexList, "renderIndexList", torch.int32, dev, (m,))
    if _rows(viewDirList, "viewDirList", 3, dev) != m:
        raise ValueError("GenerateRayPoints: viewDirList must match renderPointList")
    with torch.cuda.device(dev):
        call("qsdvr_generate_ray_points", _p(rayList), _p(originList), _p(dirList), n, float(interval),
             int(baseVolumeReso), _p(sdfPointList), _p(sdfIndexList), _p(renderPointList), _p(renderIndexList),
             _p(viewDirList), s, m, _stream(dev))
