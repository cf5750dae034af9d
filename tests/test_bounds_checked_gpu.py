"""The bounds-checked build (libqsdvr_b200_debug.so: the same sources compiled with
-DQSDVR_DEBUG_BOUNDS) in place of compute-sanitizer: every global gather, store and RED
whose index a kernel derives from geometry or caller data is checked against its buffer,
and a violation is recorded and redirected instead of faulting.

* a positive control that is in bounds by construction (a 64-float buffer declared as 32):
  the checked build catches and records the write, the product build performs it;
* the GPU parity suites run again in a child process on the checked library, and the
  autouse fixture of conftest.py fails any test after which a violation was recorded.
"""
import json
import os
import subprocess
import sys

import pytest
import torch

from conftest import ROOT

pytestmark = pytest.mark.gpu

_CONTROL = r"""
import json, sys, torch
sys.path.insert(0, sys.argv[1])
from qsdvr_b200 import _lib
buf = torch.zeros(64, dtype=torch.float32, device="cuda")
_lib.call("qsdvr_check_bounds", buf.data_ptr(), None)
print(json.dumps({"checked": _lib.bounds_checked(), "record": _lib.bounds_record(),
                  "error": _lib.device_error(), "value": float(buf[40]), "others": float(buf.sum() - buf[40])}))
"""


def _child(code_or_args, env_lib, timeout):
    env = dict(os.environ, QSDVR_B200_LIB=env_lib)
    return subprocess.run(code_or_args, cwd=ROOT, env=env, capture_output=True, text=True, timeout=timeout)


def test_product_build_writes_the_control_element():
    from qsdvr_b200 import _lib

    assert not _lib.bounds_checked()
    buf = torch.zeros(64, dtype=torch.float32, device="cuda")
    _lib.call("qsdvr_check_bounds", buf.data_ptr(), None)
    assert float(buf[40]) == 1.0 and float(buf.sum()) == 1.0
    assert _lib.bounds_record() is None
    assert _lib.device_error() & _lib.QSDVR_DEVERR_BOUNDS == 0


def test_checked_build_catches_and_records_the_control():
    from qsdvr_b200 import _lib

    out = _child([sys.executable, "-c", _CONTROL, ROOT], _lib.DEBUG_LIB_PATH, 300)
    assert out.returncode == 0, out.stderr[-2000:]
    res = json.loads(out.stdout.strip().splitlines()[-1])
    assert res["checked"] is True
    src, line, index, extent = res["record"]
    assert (src, index, extent) == ("fused.cu", 40, 32) and line > 0
    assert res["error"] & _lib.QSDVR_DEVERR_BOUNDS
    assert res["value"] == 0.0 and res["others"] == 0.0  # redirected: the buffer is untouched


def test_parity_suites_clean_under_the_checked_build():
    from qsdvr_b200 import _lib

    skip = {"test_bounds_checked_gpu.py", "test_reference_speed_gpu.py"}
    files = sorted(f for f in os.listdir(os.path.join(ROOT, "tests"))
                   if f.startswith("test_") and f.endswith("_gpu.py") and f not in skip)
    files.append("test_zz_no_alloc.py")  # the fixed-scratch RayCut, collected last
    out = _child([sys.executable, "-m", "pytest", *[os.path.join("tests", f) for f in files], "-m", "gpu", "-x", "-q",
                  "-p", "no:cacheprovider"], _lib.DEBUG_LIB_PATH, 1500)
    tail = "\n".join(out.stdout.strip().splitlines()[-15:])
    print(f"\nparity suites on the bounds-checked library: {tail.splitlines()[-1] if tail else out.stderr[-500:]}")
    assert out.returncode == 0, tail + out.stderr[-2000:]
    assert " passed" in tail and "failed" not in tail
