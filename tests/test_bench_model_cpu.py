"""The bench's algorithmic-byte model of the train kernel (the roofline numerator), on the
CPU: 64 B of quadric cells read per render sample; 64 B of SDF-cell gradient
read-modify-write for each sample whose SDF sample has a gradient (alpha > 0 on either
interval it bounds); for each active sample (alpha > 0) its render cell's normal gradient
(64 B), its 8 corner rows gathered once and its 8 gradient rows read-modify-written in L2."""
import pytest

import bench


@pytest.mark.parametrize("storage,sh,grad,active", [
    ("f32", 2, "f32", 64 + 8 * 32 * 4 + 2 * 8 * 32 * 4),
    ("bf16", 2, "f32", 64 + 8 * 32 * 2 + 2 * 8 * 32 * 4),
    ("bf16", 2, "bf16", 64 + 8 * 32 * 2 + 2 * 8 * 32 * 2),
    ("f32", 3, "f32", 64 + 8 * 64 * 4 + 2 * 8 * 64 * 4),
    ("bf16", 3, "f32", 64 + 8 * 64 * 2 + 2 * 8 * 64 * 4),
])
def test_byte_terms(storage, sh, grad, active):
    assert bench.byte_terms(storage, sh, grad) == (64, 64, active)


def test_bytes_per_sample_interpolates_with_the_active_fractions():
    # all active: the dense model (3264 B for fp32 SH 2, what every sample cost before alpha = 0
    # samples were skipped); half active with 0.51 sending an SDF-cell gradient: 1664.6 B
    assert bench.bytes_per_sample("f32", 2) == 3264
    assert bench.bytes_per_sample("f32", 2, active=0.5, sdf_grad=0.51) == pytest.approx(64 + 0.51 * 64 + 0.5 * 3136)
    assert bench.bytes_per_sample("f32", 2, active=0.0, sdf_grad=0.0) == 64


def test_reference_arm_batch_is_built_on_the_host():
    """The reference arm's batch (bench.reference_batch_cpu) comes from the oracle alone: rays
    marched by the C RayCut with packed offsets, targets rendered by the oracle, the product
    library never loaded."""
    import numpy as np

    import bench

    cfg = dict(bench.WORKLOADS["plain128"], R=16, views=3, size=40, focal=55.0)
    grid7, data, b = bench.reference_batch_cpu(cfg, 12)
    rays = b["rays"].astype(np.int64)
    assert rays.shape == (12, 4) and grid7.shape == (16 ** 3, 7) and data.shape == (17 ** 3, 32)
    assert np.array_equal(rays[:, 1], np.cumsum(rays[:, 0]) - rays[:, 0])
    assert np.array_equal(rays[:, 2], np.maximum(rays[:, 0] - 1, 0))
    assert np.isfinite(b["target"].numpy()).all() and b["target"].shape == (12, 3)
    full = dict(bench.WORKLOADS["config1"], R=16)
    _, _, fb = bench.reference_batch_cpu(full, 0)
    assert fb["rays"].shape == (100 * 100, 4) and int((fb["rays"][:, 0] >= 2).sum()) > 1000
    # a fresh process that builds such a batch never maps the product library
    import subprocess
    import sys

    code = ("import bench; cfg = dict(bench.WORKLOADS['plain128'], R=16, views=2, size=24, focal=33.0); "
            "bench.reference_batch_cpu(cfg, 4); print('libqsdvr_b200' in open('/proc/self/maps').read())")
    out = subprocess.run([sys.executable, "-c", code], cwd=bench.ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.strip().splitlines()[-1] == "False"
