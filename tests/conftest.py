import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def pytest_collection_modifyitems(config, items):
    import torch

    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(autouse=True)
def _no_out_of_range_access():
    """Under the bounds-checked library (QSDVR_B200_LIB=qsdvr_b200/libqsdvr_b200_debug.so)
    every test must end with no out-of-range access caught by the kernels' range checks."""
    yield
    from qsdvr_b200 import _lib

    if _lib._lib is None or not _lib.bounds_checked():
        return
    import torch

    if torch.cuda.is_available():
        rec = _lib.bounds_record()
        assert rec is None, f"out-of-range access caught at {rec[0]}:{rec[1]} (index {rec[2]}, extent {rec[3]})"


def load_golden(name: str):
    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        pytest.skip(f"golden fixture {name}.npz not generated yet (tests/golden/make_golden.py on a GPU)")
    return dict(np.load(path))


@pytest.fixture(scope="session")
def golden_raygen():
    return load_golden("raygen")


@pytest.fixture(scope="session")
def golden_ops():
    return load_golden("ops")


@pytest.fixture(scope="session")
def golden_pipeline():
    return load_golden("pipeline")


def rel_err(a, b):
    """max |a - b| / max |b| over finite entries (norm-wise relative error, robust to
    entries near zero).  Non-finite entries must sit at the same places in both: the
    reference's compositing backward divides by (alpha - 1) and yields NaN/inf where alpha
    rounds to 1 (kernel/render.cu:300,313); parity means reproducing exactly those."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    fa, fb = np.isfinite(a), np.isfinite(b)
    if not np.array_equal(fa, fb):
        return float("inf")
    if not fa.any():
        return 0.0
    a, b = a[fa], b[fb]
    scale = np.abs(b).max()
    return float(np.abs(a - b).max() / (scale if scale > 0 else 1.0))


def camera_from_record(rec):
    """CameraArgs from a make_golden camera record."""
    from qsdvr_b200.qsdvr import CameraArgs

    r = np.asarray(rec, np.float64)
    a = CameraArgs()
    a.width, a.height = int(r[0]), int(r[1])
    a.rotation = r[2:11]
    a.translation = r[11:14]
    a.fx, a.fy, a.cx, a.cy, a.near, a.far = (float(v) for v in r[14:20])
    a.pixelCount = a.width * a.height
    return a


def oracle_camera(args):
    import oracle.oracle as O

    return O.Camera(args.width, args.height, tuple(args.rotation), tuple(args.translation), args.fx, args.fy, args.cx,
                    args.cy, args.near, args.far)
