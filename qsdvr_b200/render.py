"""The reference's model layer (models/render.py) on top of the B200 kernels.

Same class names, constructor arguments, parameters, forward inputs and outputs as
models/render.py:8-237: six ``autograd.Function``s around the per-op kernels, the
separable ``QuadricGrid`` and the ``RenderGrid`` module.  ``mode='compat'`` (default)
reproduces the reference exactly, including its shading read of the SH coefficients;
``mode='fixed'`` uses the packed layout whose backward is the exact gradient.
"""
from __future__ import annotations

import math
from typing import Any

import torch
from torch import autograd, nn

from . import qsdvr


class GridInterpolation(autograd.Function):
    """models/render.py:8-35."""

    @staticmethod
    def forward(ctx: Any, dataGrid: torch.Tensor, pointList: torch.Tensor, indexList: torch.Tensor):
        pointCount = pointList.size(0)
        dataCount = dataGrid.size(3)
        reso = dataGrid.size(0)
        out = torch.empty((pointCount, dataCount), dtype=torch.float32, device=dataGrid.device)
        qsdvr.GridInterpolationForward(dataGrid, pointList, indexList, out, reso)
        ctx.save_for_backward(pointList, indexList)
        ctx.reso = reso
        ctx.dataCount = dataCount
        return out

    @staticmethod
    def backward(ctx: Any, gradOutput: Any):
        pointList, indexList = ctx.saved_tensors
        dataGradGrid = torch.zeros((ctx.reso, ctx.reso, ctx.reso, ctx.dataCount), dtype=torch.float32,
                                   device=pointList.device)
        qsdvr.GridInterpolationBackward(dataGradGrid, pointList, indexList, gradOutput.contiguous(), ctx.reso)
        return dataGradGrid, None, None


class Shader(autograd.Function):
    """models/render.py:38-65 (the shading mode is the fourth argument, default compat)."""

    @staticmethod
    def forward(ctx: Any, normalList: torch.Tensor, viewDirList: torch.Tensor, dataList: torch.Tensor,
                mode: str = "compat"):
        pointCount = normalList.size(0)
        out = torch.empty((pointCount, 3), dtype=torch.float32, device=dataList.device)
        specularList = torch.empty((pointCount, 3), dtype=torch.float32, device=dataList.device)
        qsdvr.ShaderForward(out, normalList, viewDirList, dataList, specularList, mode=mode)
        ctx.save_for_backward(normalList, viewDirList, dataList, specularList)
        ctx.mode = mode
        return out

    @staticmethod
    def backward(ctx: Any, gradOutput: Any):
        normalList, viewDirList, dataList, specularList = ctx.saved_tensors
        pointCount = normalList.size(0)
        normalGradList = torch.empty((pointCount, 3), dtype=torch.float32, device=dataList.device)
        dataGradList = torch.empty((pointCount, 32), dtype=torch.float32, device=dataList.device)
        qsdvr.ShaderBackward(gradOutput.contiguous(), normalList, viewDirList, dataList, specularList, normalGradList,
                             dataGradList, mode=ctx.mode)
        return normalGradList, None, dataGradList, None


class RayAggregate(autograd.Function):
    """models/render.py:68-98."""

    @staticmethod
    def forward(ctx: Any, rgbList: torch.Tensor, sdfList: torch.Tensor, rayList: torch.Tensor, logisticCoef):
        pixelCount = rayList.size(0)
        renderCount = rgbList.size(0)
        dev = rgbList.device
        out = torch.empty((pixelCount, 3), dtype=torch.float32, device=dev)
        alphaList = torch.empty(renderCount, dtype=torch.float32, device=dev)
        TList = torch.empty(renderCount, dtype=torch.float32, device=dev)
        qsdvr.RayAggregateForward(out, rgbList, sdfList, rayList, alphaList, TList, logisticCoef)
        ctx.save_for_backward(rgbList, sdfList, rayList, alphaList, TList)
        ctx.logisticCoef = logisticCoef
        return out

    @staticmethod
    def backward(ctx: Any, gradOutput: Any):
        rgbList, sdfList, rayList, alphaList, TList = ctx.saved_tensors
        dev = rgbList.device
        rgbGradList = torch.empty((rgbList.size(0), 3), dtype=torch.float32, device=dev)
        sdfGradList = torch.empty(sdfList.size(0), dtype=torch.float32, device=dev)
        qsdvr.RayAggregateBackward(gradOutput.contiguous(), rgbList, sdfList, rayList, alphaList, TList, rgbGradList,
                                   sdfGradList, ctx.logisticCoef)
        return rgbGradList, sdfGradList, None, None


class LayerToGrid(autograd.Function):
    """models/render.py:101-122."""

    @staticmethod
    def forward(ctx: Any, xLayer: torch.Tensor, yLayer: torch.Tensor, zLayer: torch.Tensor, offset: torch.Tensor,
                device=None):
        reso = xLayer.size(0)
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        out = torch.empty((reso, reso, reso, 7), dtype=torch.float32, device=dev)
        qsdvr.LayerToGridForward(out, xLayer.detach(), yLayer.detach(), zLayer.detach(), offset.detach())
        ctx.reso = reso
        ctx.layer_device = xLayer.device
        return out

    @staticmethod
    def backward(ctx: Any, gradOutput: Any):
        reso = ctx.reso
        dev = ctx.layer_device
        xLayer = torch.empty(reso, dtype=torch.float32, device=dev)
        yLayer = torch.empty(reso, dtype=torch.float32, device=dev)
        zLayer = torch.empty(reso, dtype=torch.float32, device=dev)
        offset = torch.empty(4, dtype=torch.float32, device=dev)
        qsdvr.LayerToGridBackward(gradOutput.contiguous(), xLayer, yLayer, zLayer, offset)
        return xLayer, yLayer, zLayer, offset, None


class SampleSDF(autograd.Function):
    """models/render.py:125-146."""

    @staticmethod
    def forward(ctx: Any, sdfGrid: torch.Tensor, pointList: torch.Tensor, indexList: torch.Tensor):
        out = torch.empty(pointList.size(0), dtype=torch.float32, device=sdfGrid.device)
        qsdvr.SampleSDFForward(out, sdfGrid, pointList, indexList, sdfGrid.size(0))
        ctx.save_for_backward(sdfGrid, pointList, indexList)
        ctx.reso = sdfGrid.size(0)
        return out

    @staticmethod
    def backward(ctx: Any, gradOutput: Any):
        sdfGrid, pointList, indexList = ctx.saved_tensors
        sdfGradGrid = torch.zeros((ctx.reso, ctx.reso, ctx.reso, 7), dtype=torch.float32, device=sdfGrid.device)
        qsdvr.SampleSDFBackward(gradOutput.contiguous(), sdfGrid, pointList, indexList, sdfGradGrid, ctx.reso)
        return sdfGradGrid, None, None


class SampleNormal(autograd.Function):
    """models/render.py:149-169."""

    @staticmethod
    def forward(ctx: Any, sdfGrid: torch.Tensor, pointList: torch.Tensor, indexList: torch.Tensor):
        out = torch.empty((pointList.size(0), 3), dtype=torch.float32, device=sdfGrid.device)
        qsdvr.SampleNormalForward(out, sdfGrid, pointList, indexList)
        ctx.save_for_backward(sdfGrid, pointList, indexList)
        ctx.reso = sdfGrid.size(0)
        return out

    @staticmethod
    def backward(ctx: Any, gradOutput: Any):
        sdfGrid, pointList, indexList = ctx.saved_tensors
        sdfGradGrid = torch.zeros((ctx.reso, ctx.reso, ctx.reso, 7), dtype=torch.float32, device=sdfGrid.device)
        qsdvr.SampleNormalBackward(gradOutput.contiguous(), sdfGrid, pointList, indexList, sdfGradGrid)
        return sdfGradGrid, None, None


class QuadricGrid(nn.Module):
    """models/render.py:172-206: separable layers (CPU parameters, as in the reference)."""

    def __init__(self, reso: int = 128, layer_device: str = "cpu"):
        super().__init__()
        self.reso = reso
        self.xLayer = nn.Parameter(torch.ones(reso, dtype=torch.float32, device=layer_device))
        self.yLayer = nn.Parameter(torch.ones(reso, dtype=torch.float32, device=layer_device))
        self.zLayer = nn.Parameter(torch.ones(reso, dtype=torch.float32, device=layer_device))
        self.offset = torch.zeros(4, dtype=torch.float32, device=layer_device)
        self.init_as_sphere()
        self.offset = nn.Parameter(self.offset)

    def init_as_sphere(self, radius=1.0):
        """models/render.py:187-192 (the reference's constants, unchanged)."""
        c = -self.reso
        with torch.no_grad():
            self.offset[0] = -2 * c
            self.offset[1] = -2 * c
            self.offset[2] = -2 * c
            self.offset[3] = math.sqrt(3 * c * c)

    def forward(self, renderPointList, renderIndexList, sdfPointList, sdfIndexList):
        sdfGrid = LayerToGrid.apply(self.xLayer, self.yLayer, self.zLayer, self.offset, renderPointList.device)
        sdfList = SampleSDF.apply(sdfGrid, sdfPointList, sdfIndexList)
        normalList = SampleNormal.apply(sdfGrid, renderPointList, renderIndexList)
        return sdfList, normalList


class RenderGrid(nn.Module):
    """models/render.py:209-237: forward(input dict) -> [N,3] ray colours."""

    def __init__(self, reso: int = 128, logisticCoef: float = 5, mode: str = "compat", device="cuda"):
        super().__init__()
        self.quadricGrid = QuadricGrid(reso)
        self.reso = reso
        self.mode = mode
        data = torch.zeros((reso + 1, reso + 1, reso + 1, 32), dtype=torch.float32, device=device)
        self.logisticCoef = logisticCoef
        data[..., 31] = 1
        data[..., 30] = 0.1
        data[..., 27:30] = 1
        data[..., 0:3] = 0.5
        self.renderData = nn.Parameter(data)

    def forward(self, input):
        sdfList, normalList = self.quadricGrid.forward(input["renderPointList"], input["renderIndexList"],
                                                       input["sdfPointList"], input["sdfIndexList"])
        index = input["renderIndexList"]
        if self.mode == "fixed":
            index = vertex_index(index, self.reso)
        datalist = GridInterpolation.apply(self.renderData, input["renderPointList"], index)
        rgbList = Shader.apply(normalList, input["viewDirList"], datalist, self.mode)
        return RayAggregate.apply(rgbList, sdfList, input["rayList"], self.logisticCoef)

    def set_logisticCoef(self, logisticCoef):
        self.logisticCoef = logisticCoef


def vertex_index(cell_index: torch.Tensor, reso: int) -> torch.Tensor:
    """Base vertex x + y(R+1) + z(R+1)^2 of cell x + yR + zR^2 (the fixed-mode addressing)."""
    i = cell_index.long()
    x, y, z = i % reso, (i // reso) % reso, i // (reso * reso)
    return (x + y * (reso + 1) + z * (reso + 1) * (reso + 1)).to(torch.int32)
