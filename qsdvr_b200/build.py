"""Build libqsdvr_b200.so in-tree with nvcc for sm_100a (no GPU needed to compile).

Each translation unit under csrc/ is compiled to an object in qsdvr_b200/_build/ (in
parallel, skipped when up to date) and linked into qsdvr_b200/libqsdvr_b200.so with the
static CUDA runtime, so the library does not depend on which libcudart torch loaded.

build(bounds_checked=True) compiles the same sources with -DQSDVR_DEBUG_BOUNDS into
qsdvr_b200/_build/bounds/ and qsdvr_b200/libqsdvr_b200_debug.so: every global access whose
index a kernel derives is range-checked, and a violation is recorded, not faulted
(select it with QSDVR_B200_LIB, see _lib.py).
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libqsdvr_b200.so")
DEBUG_LIB = os.path.join(PKG, "libqsdvr_b200_debug.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, extra: list[str], verbose: bool, obj_dir: str = OBJ) -> str:
    obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _headers_mtime()):
        return obj
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return obj


def build(verbose: bool = False, extra: list[str] | None = None, bounds_checked: bool = False) -> str:
    obj_dir = os.path.join(OBJ, "bounds") if bounds_checked else OBJ
    lib = DEBUG_LIB if bounds_checked else LIB
    flags = [*(extra or []), *(["-DQSDVR_DEBUG_BOUNDS"] if bounds_checked else [])]
    os.makedirs(obj_dir, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, flags, verbose, obj_dir), srcs))
    if not os.path.exists(lib) or os.path.getmtime(lib) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", lib, *objs, "-cudart", "static"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, bounds_checked="--bounds" in sys.argv))
