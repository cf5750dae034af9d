"""Per-camera ray tables and per-step sample lists (datasets/utils.py:6-56).

``Camera`` keeps the reference's interface: ``GenerateRayPoints(mask)`` runs RayCut once
and keeps the masked rays; ``GetRayPoints()`` allocates the sample lists and fills them
with GenerateRayPoints.  Everything stays on the device (the reference moves the ray
tables to the host after RayCut and back on every call).
"""
from __future__ import annotations

import struct
import zlib

import numpy as np
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

    def GenerateRayPoints(self, mask: torch.Tensor, order: str = "pixels", tile: int = 8):
        """datasets/utils.py:42-56: RayCut over all pixels, then keep the masked rays.

        ``order="pixels"`` keeps the reference's row-major pixel order.  ``order="tiles"``
        lists the rays tile by tile (``tile`` x ``tile`` pixels, tiles and the pixels inside
        them row-major), so that rays adjacent in the list are adjacent on the image; each
        ray keeps its RayCut record, and ``pixel_index`` maps the list back to pixels."""
        if order not in ("pixels", "tiles"):
            raise ValueError(f"order must be 'pixels' or 'tiles', got {order!r}")
        dev = self.device
        P = self.args.pixelCount
        rays = torch.zeros((P, 4), dtype=torch.int32, device=dev)
        origin = torch.zeros((P, 3), dtype=torch.float32, device=dev)
        direction = torch.zeros((P, 3), dtype=torch.float32, device=dev)
        qsdvr.RayCut(self.args, mask, rays, origin, direction, self.interval)
        m = mask.reshape(-1)[:P].to(dev, torch.bool)
        self.mask = m
        pix = torch.nonzero(m).reshape(-1)
        if order == "tiles":
            pix = tile_order(pix, self.args.width, tile)
        self.pixel_index = pix
        self.rayList = rays[pix].contiguous()
        self.originList = origin[pix].contiguous()
        self.dirList = direction[pix].contiguous()

    def whole_image(self, colors: torch.Tensor) -> torch.Tensor:
        """datasets/nerf_dataset.py:92-96 (get_whole_image): the rays' colours [N, 3] (in the
        order of rayList) scattered into a [height, width, 3] frame, zero where the mask is
        off (on the colours' device)."""
        a = self.args
        pix = self.pixel_index.to(colors.device)
        if colors.shape != (pix.numel(), 3):
            raise ValueError(f"colors must be [{pix.numel()}, 3], got {tuple(colors.shape)}")
        img = torch.zeros((a.height * a.width, 3), dtype=colors.dtype, device=colors.device)
        img[pix] = colors
        return img.reshape(a.height, a.width, 3)


def tile_order(pixels: torch.Tensor, width: int, tile: int = 8) -> torch.Tensor:
    """``pixels`` (row-major indices of an image ``width`` wide) listed tile by tile: tiles of
    ``tile`` x ``tile`` pixels in row-major order, the pixels of a tile row-major inside it."""
    y, x = pixels // width, pixels % width
    ntx = (width + tile - 1) // tile
    key = ((y // tile) * ntx + x // tile) * (tile * tile) + (y % tile) * tile + (x % tile)
    return pixels[torch.argsort(key)]


def save_png(path: str, image) -> None:
    """Write an [H, W, 3] image with values in [0, 1] as an 8-bit RGB PNG, as test.py:41-44
    does with imageio ((img * 255).clip(0, 255) as uint8), using only the standard library."""
    img = image.detach().cpu().numpy() if isinstance(image, torch.Tensor) else np.asarray(image)
    if img.ndim != 3 or img.shape[2] != 3:
        raise ValueError("image must be [H, W, 3]")
    px = (img * 255).clip(0, 255).astype(np.uint8)
    h, w = px.shape[:2]
    raw = b"".join(b"\x00" + px[y].tobytes() for y in range(h))  # filter type 0 per row

    def chunk(tag: bytes, body: bytes) -> bytes:
        return struct.pack(">I", len(body)) + tag + body + struct.pack(">I", zlib.crc32(tag + body) & 0xFFFFFFFF)

    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n")
        f.write(chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)))
        f.write(chunk(b"IDAT", zlib.compress(raw, 6)))
        f.write(chunk(b"IEND", b""))
