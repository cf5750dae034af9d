"""qsdvr_ray_cut_noalloc: RayCut for callers that cannot allocate device memory.

Some callers own all their device memory up front (their own pool or arena) or hand a
plugin nothing but input and output buffers, so they cannot supply the workspace that
qsdvr_ray_cut needs.  The no-allocation variant keeps its scan scratch in a fixed array
inside the library.  This test calls it through the C ABI twice in a row, on two different
cameras, and checks every output against the workspace entry point (counts, offsets and
directions are integer / bit-exact work, so the comparison is exact), at exactly the size
limit (2048 x 2048, every slot of the fixed array in use) against the same entry point, and
with no pixels (totals zero).  It also checks the size limit is enforced.  It lives in a file
of its own that pytest collects last.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _lib():
    from qsdvr_b200 import _lib as L

    lib = L.lib()
    fn = lib.qsdvr_ray_cut_noalloc
    fn.argtypes = [ctypes.POINTER(L.Camera), L.P, L.P, L.P, L.P, L.F32, L.U32, L.P, L.P]
    fn.restype = ctypes.c_int
    return L, lib


def _buffers(P):
    return (torch.zeros((P, 4), dtype=torch.int32, device=DEV), torch.zeros((P, 3), device=DEV),
            torch.zeros((P, 3), device=DEV), torch.zeros(2, dtype=torch.int32, device=DEV))


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _with_workspace(L, cam, mask, P, interval, stream):
    rays, origin, direction, totals = _buffers(P)
    ws = torch.empty(L.size("qsdvr_ray_cut_workspace_size", P), dtype=torch.uint8, device=DEV)
    L.call("qsdvr_ray_cut", ctypes.byref(cam), _p(mask), _p(rays), _p(origin), _p(direction), interval, P, _p(totals),
           _p(ws), ws.numel(), stream)
    return rays, origin, direction, totals


def _no_alloc(L, lib, cam, mask, P, interval, stream):
    rays, origin, direction, totals = _buffers(P)
    st = lib.qsdvr_ray_cut_noalloc(ctypes.byref(cam), _p(mask), _p(rays), _p(origin), _p(direction), interval, P,
                                   _p(totals), stream)
    assert st == 0, lib.qsdvr_last_error().decode()
    return rays, origin, direction, totals


def test_ray_cut_noalloc_matches_workspace_entry_point():
    from qsdvr_b200 import scenes

    L, lib = _lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    cases = [((0.3, -4.0, 0.5), 320, 240, 4.0 / 256, 0.8), ((2.9, 2.2, 1.6), 512, 384, 4.0 / 64, 0.6)]
    for pos, w, h, interval, density in cases:  # two calls in a row, different sizes and masks
        args = scenes.look_at(pos, w, h, 1.4 * w, 2.0, 6.0)
        cam = args.to_c()
        P = w * h
        gen = torch.Generator().manual_seed(w)
        mask = (torch.rand(P, generator=gen) < density).to(torch.uint8).to(DEV)
        want = _with_workspace(L, cam, mask, P, interval, stream)
        got = _no_alloc(L, lib, cam, mask, P, interval, stream)
        torch.cuda.synchronize()
        for a, b in zip(got, want):
            assert torch.equal(a, b)
        assert int(got[3][0]) > 0


def test_ray_cut_noalloc_rejects_oversized_pixel_count():
    L, lib = _lib()
    cam = L.Camera()
    cam.width, cam.height = 4096, 4096
    dummy = torch.zeros(16, dtype=torch.int32, device=DEV)
    limit = 4194304
    st = lib.qsdvr_ray_cut_noalloc(ctypes.byref(cam), _p(dummy), _p(dummy), _p(dummy), _p(dummy), 0.01, limit + 1,
                                   _p(dummy), None)
    assert st == 1
    assert "exceeds the fixed scratch limit" in lib.qsdvr_last_error().decode()


def test_ray_cut_noalloc_at_the_limit_and_empty():
    from qsdvr_b200 import scenes

    L, lib = _lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    w = h = 2048
    P = w * h
    assert P == 4194304  # QSDVR_RAY_CUT_NOALLOC_MAX_PIXELS: all scan blocks of the fixed array
    cam = scenes.look_at((1.1, -3.6, 1.3), w, h, 1.2 * w, 2.0, 6.0).to_c()
    mask = (torch.rand(P, generator=torch.Generator().manual_seed(5)) < 0.7).to(torch.uint8).to(DEV)
    want = _with_workspace(L, cam, mask, P, 4.0 / 128, stream)
    got = _no_alloc(L, lib, cam, mask, P, 4.0 / 128, stream)
    torch.cuda.synchronize()
    for a, b in zip(got, want):
        assert torch.equal(a, b)
    assert int(got[3][0]) > 0
    rays, origin, direction, totals = _buffers(4)
    totals.fill_(7)
    st = lib.qsdvr_ray_cut_noalloc(ctypes.byref(cam), _p(mask), _p(rays), _p(origin), _p(direction), 4.0 / 128, 0,
                                   _p(totals), stream)
    assert st == 0, lib.qsdvr_last_error().decode()
    torch.cuda.synchronize()
    assert totals.tolist() == [0, 0]
