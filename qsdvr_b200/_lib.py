"""ctypes binding of libqsdvr_b200.so (the C ABI declared in include/qsdvr_b200.h).

The library is the only compute path: if it is missing or fails to load, every entry
point raises.  There is no CPU or PyTorch fallback.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# QSDVR_B200_LIB selects another build of the library, e.g. DEBUG_LIB_PATH, the bounds-checked
# variant of the same sources (every derived index range-checked; violations recorded).
LIB_PATH = os.environ.get("QSDVR_B200_LIB") or os.path.join(_HERE, "libqsdvr_b200.so")
DEBUG_LIB_PATH = os.path.join(_HERE, "libqsdvr_b200_debug.so")

P = ctypes.c_void_p
U32 = ctypes.c_uint32
U64 = ctypes.c_uint64
F32 = ctypes.c_float
I32 = ctypes.c_int
SZ = ctypes.c_size_t

OK = 0
MODE_COMPAT = 0
MODE_FIXED = 1

DEVERR_INDEX = 1
DEVERR_CAPACITY = 2
DEVERR_RAY = 4
DEVERR_TIMEOUT = 8
DEVERR_BOUNDS = 16


class Camera(ctypes.Structure):
    """qsdvr_camera (include/qsdvr_b200.h)."""
    _fields_ = [("width", U32), ("height", U32), ("rotation", F32 * 9), ("translation", F32 * 3),
                ("fx", F32), ("fy", F32), ("cx", F32), ("cy", F32), ("near_depth", F32), ("far_depth", F32)]


# name -> argtypes; every function returns int status except where noted
_SIGS = {
    "qsdvr_version": [],
    "qsdvr_device_error": [P, I32, P],
    "qsdvr_bounds_checked": [],
    "qsdvr_bounds_record": [P, I32, P],
    "qsdvr_check_bounds": [P, P],
    "qsdvr_ray_cut": [ctypes.POINTER(Camera), P, P, P, P, F32, U32, P, P, SZ, P],
    "qsdvr_generate_ray_points": [P, P, P, U32, F32, U32, P, P, P, P, P, U64, U64, P],
    "qsdvr_layer_to_grid_forward": [P, P, P, P, P, U32, P, SZ, P],
    "qsdvr_layer_to_grid_backward": [P, U32, P, P, P, P, P, SZ, P],
    "qsdvr_sample_sdf_forward": [P, P, P, P, U64, F32, U64, P],
    "qsdvr_sample_sdf_backward": [P, P, P, P, P, U64, F32, U64, P],
    "qsdvr_sample_normal_forward": [P, P, P, P, U64, U64, P],
    "qsdvr_sample_normal_backward": [P, P, P, P, P, U64, U64, P],
    "qsdvr_grid_interpolation_forward": [P, P, P, P, U64, U32, U64, P],
    "qsdvr_grid_interpolation_backward": [P, P, P, P, U64, U32, U64, P],
    "qsdvr_shader_forward": [P, P, P, P, P, U64, I32, P],
    "qsdvr_shader_backward": [P, P, P, P, P, P, P, U64, I32, P],
    "qsdvr_ray_aggregate_forward": [P, P, P, P, P, P, U32, F32, U64, U64, P],
    "qsdvr_ray_aggregate_backward": [P, P, P, P, P, P, P, P, U32, F32, U64, U64, P],
}
_SIZE_FNS = {
    "qsdvr_ray_cut_workspace_size": [U32],
    "qsdvr_layer_to_grid_workspace_size": [U32],
}

_lib = None


class QsdvrError(RuntimeError):
    """A non-OK status from the C ABI."""

    def __init__(self, fn: str, code: int, msg: str):
        super().__init__(f"{fn} failed with status {code}: {msg}")
        self.code = code


def extra_signatures(sigs: dict, size_fns: dict | None = None):
    """Register further entry points (used by modules that add C-ABI functions)."""
    _SIGS.update(sigs)
    if size_fns:
        _SIZE_FNS.update(size_fns)
    if _lib is not None:
        _declare(_lib)


def _declare(lib):
    for name, args in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = I32
    for name, args in _SIZE_FNS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = SZ
    lib.qsdvr_last_error.argtypes = []
    lib.qsdvr_last_error.restype = ctypes.c_char_p


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"qsdvr_b200: {LIB_PATH} is missing; build it with "
                               "`python -c 'import __graft_entry__ as g; g.build()'` or qsdvr_b200/build.py")
        handle = ctypes.CDLL(LIB_PATH)
        _declare(handle)
        _lib = handle
    return _lib


def call(name: str, *args) -> None:
    """Call a status-returning entry point and raise QsdvrError on failure."""
    status = getattr(lib(), name)(*args)
    if status != OK:
        raise QsdvrError(name, status, lib().qsdvr_last_error().decode(errors="replace"))


def size(name: str, *args) -> int:
    return int(getattr(lib(), name)(*args))


# bits of the device error word (include/qsdvr_b200.h)
QSDVR_DEVERR_INDEX, QSDVR_DEVERR_CAPACITY, QSDVR_DEVERR_RAY, QSDVR_DEVERR_TIMEOUT = 1, 2, 4, 8
QSDVR_DEVERR_BOUNDS = 16
# source files of qsdvr_bounds_record's first field
BOUNDS_SOURCES = {1: "camera.cu", 2: "surface.cu", 3: "render_ops.cu", 4: "fused.cu", 5: "optim.cu",
                  6: "gradcheck.cu", 7: "proposal.cu"}


def device_error(stream=None, clear: bool = True) -> int:
    """Read (and by default clear) the device error word; synchronises the stream."""
    w = ctypes.c_uint32(0)
    call("qsdvr_device_error", ctypes.byref(w), int(clear), stream)
    return int(w.value)


def bounds_checked() -> bool:
    """True when the loaded library is the bounds-checked build."""
    return bool(lib().qsdvr_bounds_checked())


def bounds_record(stream=None, clear: bool = True):
    """The first out-of-range access the bounds-checked build caught since the last clear, as
    (source file, line, element index, buffer extent), or None; synchronises the stream."""
    rec = (ctypes.c_uint64 * 4)()
    call("qsdvr_bounds_record", rec, int(clear), stream)
    if rec[0] == 0:
        return None
    return BOUNDS_SOURCES.get(int(rec[0]), str(int(rec[0]))), int(rec[1]), int(rec[2]), int(rec[3])
