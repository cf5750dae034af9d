"""C-ABI library: loads, exports every symbol include/qsdvr_b200.h declares, and the host
side validates arguments before touching a GPU.  CPU only (no compute calls)."""
import ctypes
import os
import re

import numpy as np
import pytest
import torch

from conftest import ROOT

HEADERS = [os.path.join(ROOT, "include", h) for h in sorted(os.listdir(os.path.join(ROOT, "include")))
           if h.endswith(".h")]


def declared_functions():
    names = []
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"\b(qsdvr_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "qsdvr_ray_cut" in names and "qsdvr_ray_aggregate_backward" in names
    assert len(names) >= 18


def test_library_exports_every_declared_symbol():
    from qsdvr_b200 import _lib

    lib = _lib.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.qsdvr_version() >= 100
    assert lib.qsdvr_bounds_checked() == 0  # the product build
    assert _lib.bounds_record() is None  # it keeps no record (and needs no GPU to say so)


def test_bounds_checked_build_exports_the_same_symbols():
    """libqsdvr_b200_debug.so (the same sources with -DQSDVR_DEBUG_BOUNDS) is a drop-in for the
    product library: the same entry points, and it reports itself as range-checked."""
    from qsdvr_b200 import _lib

    assert os.path.exists(_lib.DEBUG_LIB_PATH), "build() compiles the bounds-checked library too"
    dbg = ctypes.CDLL(_lib.DEBUG_LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(dbg, n)]
    assert not missing, missing
    assert dbg.qsdvr_bounds_checked() == 1
    assert dbg.qsdvr_version() == _lib.lib().qsdvr_version()


def test_workspace_size_queries():
    from qsdvr_b200 import _lib

    assert _lib.size("qsdvr_ray_cut_workspace_size", 640000) >= 8 * (640000 // 256)
    assert _lib.size("qsdvr_layer_to_grid_workspace_size", 256) == 6 * 256 * 4


def test_invalid_arguments_return_status_without_gpu():
    """Argument checks happen on the host and return a status (no kernel is launched)."""
    from qsdvr_b200 import _lib

    with pytest.raises(_lib.QsdvrError) as e:
        _lib.call("qsdvr_sample_sdf_forward", None, None, None, None, 10, 8.0, 512, None)
    assert e.value.code == 1 and "null pointer" in str(e.value)
    with pytest.raises(_lib.QsdvrError) as e:
        _lib.call("qsdvr_layer_to_grid_forward", ctypes.c_void_p(16), ctypes.c_void_p(16), ctypes.c_void_p(16),
                  ctypes.c_void_p(16), ctypes.c_void_p(16), 0, None, 0, None)
    assert e.value.code == 1
    cam = _lib.Camera()
    cam.width, cam.height = 4, 4
    with pytest.raises(_lib.QsdvrError) as e:
        _lib.call("qsdvr_ray_cut", ctypes.byref(cam), ctypes.c_void_p(16), ctypes.c_void_p(16), ctypes.c_void_p(16),
                  ctypes.c_void_p(16), 0.1, 16, ctypes.c_void_p(16), ctypes.c_void_p(16), 0, None)
    assert e.value.code == 3  # workspace too small


def test_dropin_rejects_cpu_and_wrong_dtypes():
    from qsdvr_b200 import qsdvr

    x = torch.zeros(10, 3)
    with pytest.raises(ValueError):
        qsdvr.SampleSDFForward(torch.zeros(10), torch.zeros(8, 7), x, torch.zeros(10, dtype=torch.int32), 2.0)
    with pytest.raises(TypeError):
        qsdvr.ShaderForward(x, x, x, torch.zeros(10, 32, dtype=torch.float64), x)


def test_camera_args_fields():
    from qsdvr_b200.qsdvr import CameraArgs

    a = CameraArgs()
    a.rotation = [1, 0, 0, 0, 1, 0, 0, 0, 1]
    a.translation = (0.5, 1.5, 2.5)
    assert a.rotation.dtype == np.float32 and a.rotation.shape == (9,)
    c = a.to_c()
    assert c.rotation[4] == 1.0 and c.translation[2] == 2.5
    a.rotation = [1, 2]
    with pytest.raises(ValueError):
        a.to_c()


def test_whole_image_and_png(tmp_path):
    """Image assembly (datasets/nerf_dataset.py:92-96) and the PNG writer, on the CPU: the
    masked rays' colours land at their pixels, zeros elsewhere; the PNG decodes back to the
    same 8-bit pixels."""
    import struct
    import zlib

    import numpy as np
    import torch

    from qsdvr_b200.camera import Camera, save_png
    from qsdvr_b200.qsdvr import CameraArgs

    a = CameraArgs()
    a.width, a.height = 5, 3
    cam = Camera(a, device="cpu")
    mask = torch.zeros(15, dtype=torch.bool)
    mask[[0, 4, 7, 14]] = True
    cam.mask = mask
    cam.pixel_index = torch.nonzero(mask).reshape(-1)
    colors = torch.tensor([[0.1, 0.2, 0.3], [1.0, 0.0, 0.5], [0.25, 0.75, 1.5], [-0.2, 0.6, 0.9]])
    img = cam.whole_image(colors)
    assert img.shape == (3, 5, 3)
    flat = img.reshape(-1, 3)
    assert torch.equal(flat[mask], colors) and not flat[~mask].any()
    with pytest.raises(ValueError):
        cam.whole_image(colors[:3])
    path = tmp_path / "frame.png"
    save_png(str(path), img)
    data = path.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    w, h = struct.unpack(">II", data[16:24])
    assert (w, h) == (5, 3)
    i = data.index(b"IDAT")
    n = struct.unpack(">I", data[i - 4:i])[0]
    raw = zlib.decompress(data[i + 4:i + 4 + n])
    rows = np.frombuffer(raw, np.uint8).reshape(3, 1 + 5 * 3)
    assert not rows[:, 0].any()
    want = (img.numpy() * 255).clip(0, 255).astype(np.uint8).reshape(3, 15)
    assert np.array_equal(rows[:, 1:], want)


def test_tile_order():
    """Rays listed tile by tile: the first 64 of a 20 x 12 image are its top-left 8 x 8 tile,
    row-major; partial edge tiles follow in row-major tile order; nothing is lost."""
    import torch

    from qsdvr_b200.camera import tile_order

    w, h = 20, 12
    pix = torch.arange(w * h)
    out = tile_order(pix, w, 8)
    assert torch.equal(out.sort().values, pix)
    assert torch.equal(out[:64], torch.tensor([y * w + x for y in range(8) for x in range(8)]))
    assert torch.equal(out[64:128], torch.tensor([y * w + x for y in range(8) for x in range(8, 16)]))
    assert torch.equal(out[128:160], torch.tensor([y * w + x for y in range(8) for x in range(16, 20)]))
    masked = pix[pix % 3 == 0]
    assert torch.equal(tile_order(masked, w, 8).sort().values, masked)
