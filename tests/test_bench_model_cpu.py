"""The bench's algorithmic-byte model of the train kernel (the roofline numerator), on the
CPU: 192 B of quadric cells per render sample, plus for each active sample (alpha > 0) its
8 corner rows gathered once and its 8 gradient rows read-modify-written in L2."""
import pytest

import bench


@pytest.mark.parametrize("storage,sh,grad,every,active", [
    ("f32", 2, "f32", 192, 8 * 32 * 4 + 2 * 8 * 32 * 4),
    ("bf16", 2, "f32", 192, 8 * 32 * 2 + 2 * 8 * 32 * 4),
    ("bf16", 2, "bf16", 192, 8 * 32 * 2 + 2 * 8 * 32 * 2),
    ("f32", 3, "f32", 192, 8 * 64 * 4 + 2 * 8 * 64 * 4),
    ("bf16", 3, "f32", 192, 8 * 64 * 2 + 2 * 8 * 64 * 4),
])
def test_byte_terms(storage, sh, grad, every, active):
    assert bench.byte_terms(storage, sh, grad) == (every, active)


def test_bytes_per_sample_interpolates_with_the_active_fraction():
    # all active: the dense model (3264 B for fp32 SH 2, what every sample cost before alpha = 0
    # samples were skipped); the config-3 scene's 0.50 active: 1728 B
    assert bench.bytes_per_sample("f32", 2) == 3264
    assert bench.bytes_per_sample("f32", 2, active=0.5) == 1728
    assert bench.bytes_per_sample("f32", 2, active=0.0) == 192
