"""Per-camera ray tables and per-step sample lists (datasets/utils.py:6-56).

``Camera`` keeps the reference's interface: ``GenerateRayPoints(mask)`` runs RayCut once
and keeps the masked rays; ``GetRayPoints()`` allocates the sample lists and fills them
with GenerateRayPoints.  Everything stays on the device (the reference moves the ray
tables to the host after RayCut and back on every call).
"""
from __future__ import annotations

import torch

from . import qsdvr
from .qsdvr import CameraArgs


class Camera:
    """datasets/utils.py:6-56."""

    def __init__(self, args: CameraArgs, interval: float = 0.03, reso: int = 128, device="cuda"):
        self.args = args
        self.args.pixelCount = args.width * args.height
        self.interval = interval
        self.reso = reso
        self.device = torch.device(device)

    def GetRayPoints(self):
        """datasets/utils.py:16-40: the input dict of RenderGrid.forward."""
        dev = self.device
        a = self.args
        d = {
            "rayList": self.rayList,
            "sdfPointList": torch.zeros((a.sdfCount, 3), dtype=torch.float32, device=dev),
            "sdfIndexList": torch.zeros(a.sdfCount, dtype=torch.int32, device=dev),
            "renderPointList": torch.zeros((a.renderCount, 3), dtype=torch.float32, device=dev),
            "renderIndexList": torch.zeros(a.renderCount, dtype=torch.int32, device=dev),
            "viewDirList": torch.zeros((a.renderCount, 3), dtype=torch.float32, device=dev),
        }
        qsdvr.GenerateRayPoints(a, d["sdfPointList"], d["sdfIndexList"], d["renderPointList"], d["renderIndexList"],
                                d["viewDirList"], d["rayList"], self.originList, self.dirList, self.interval,
                                self.reso)
        return d

    def GenerateRayPoints(self, mask: torch.Tensor):
        """datasets/utils.py:42-56: RayCut over all pixels, then keep the masked rays."""
        dev = self.device
        P = self.args.pixelCount
        rays = torch.zeros((P, 4), dtype=torch.int32, device=dev)
        origin = torch.zeros((P, 3), dtype=torch.float32, device=dev)
        direction = torch.zeros((P, 3), dtype=torch.float32, device=dev)
        qsdvr.RayCut(self.args, mask, rays, origin, direction, self.interval)
        m = mask.reshape(-1)[:P].to(dev, torch.bool)
        self.rayList = rays[m].contiguous()
        self.originList = origin[m].contiguous()
        self.dirList = direction[m].contiguous()
