"""ORACLE build recipe — compiles the unmodified reference (QSDVR) into ``oracle/_ref/``.

Test infrastructure only.  The reference is a PyTorch CUDA extension built from
kernel/qsdvr.cpp, kernel/camera.cu, kernel/render.cu, kernel/surface.cu with include/
(setup.py:4-15).  This recipe does not run the reference's setup.py: it compiles those
same four files, where they lie in the reference tree, with torch's extension builder and
the flags setup.py would get (torch defaults, no extra options), for sm_100 so it runs on
a B200.  The result, ``oracle/_ref/qsdvr_ref*.so``, is imported by tests and by
``tests/golden/make_golden.py`` as the parity oracle.  Nothing is copied out of the
reference tree.

Usage:  python oracle/build_ref.py [REFERENCE_ROOT]
"""
from __future__ import annotations

import glob
import importlib.util
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# where the reference sources lie in this build container; QSDVR_REFERENCE_ROOT or the
# command-line argument names another tree
DEFAULT_ROOT = os.environ.get("QSDVR_REFERENCE_ROOT", "/root/reference")
SOURCES = ("kernel/qsdvr.cpp", "kernel/camera.cu", "kernel/render.cu", "kernel/surface.cu")


def built_path() -> str | None:
    hits = sorted(glob.glob(os.path.join(OUT, "qsdvr_ref*.so")))
    return hits[0] if hits else None


def build(root: str = DEFAULT_ROOT, verbose: bool = False) -> str | None:
    """Compile the reference if its sources are present; returns the .so path or None."""
    srcs = [os.path.join(root, s) for s in SOURCES]
    if not all(os.path.exists(s) for s in srcs):
        return built_path()
    newest = max(os.path.getmtime(s) for s in srcs)
    have = built_path()
    if have and os.path.getmtime(have) >= newest:
        return have
    os.makedirs(OUT, exist_ok=True)
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0")
    os.environ.setdefault("MAX_JOBS", "4")
    from torch.utils.cpp_extension import load

    load(name="qsdvr_ref", sources=srcs, extra_include_paths=[os.path.join(root, "include")],
         build_directory=OUT, verbose=verbose, is_python_module=True)
    for junk in glob.glob(os.path.join(OUT, "*.o")) + glob.glob(os.path.join(OUT, ".ninja*")):
        try:
            os.remove(junk)
        except OSError:
            pass
    return built_path()


def load_reference():
    """Import the prebuilt reference module (``qsdvr_ref``) or return None if absent."""
    path = built_path()
    if path is None:
        return None
    import torch  # noqa: F401  (the extension links against libtorch)

    if "qsdvr_ref" in sys.modules:
        return sys.modules["qsdvr_ref"]
    spec = importlib.util.spec_from_file_location("qsdvr_ref", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    sys.modules["qsdvr_ref"] = mod
    return mod


def clear_cuda_error() -> int:
    """Consume a pending CUDA runtime error (returns its code).

    The reference's LayerToGridBackward (kernel/surface.cu:255,282) copies R floats from a
    1-float device allocation; that cudaMemcpy fails with cudaErrorInvalidValue, leaves the
    offset[3] gradient unwritten, and the error would surface at torch's next launch check.
    """
    import ctypes

    rt = ctypes.CDLL("libcudart.so.12")
    rt.cudaGetLastError.restype = ctypes.c_int
    return int(rt.cudaGetLastError())


def reference_layer_to_grid_backward(ref, grad7, reso: int):
    """Run the reference's LayerToGridBackward safely.  Returns CPU (x, y, z, offset[0:3]);
    the reference never produces offset[3] (see clear_cuda_error)."""
    import torch

    x, y, z = torch.empty(reso), torch.empty(reso), torch.empty(reso)
    off = torch.zeros(reso + 3)  # it writes R floats starting at offset[3]
    torch.cuda.synchronize()
    ref.LayerToGridBackward(grad7.contiguous(), x, y, z, off)
    torch.cuda.synchronize()
    clear_cuda_error()
    return x, y, z, off[:3].clone()


if __name__ == "__main__":
    p = build(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_ROOT, verbose=True)
    print(p if p else "reference sources not found; nothing built")
