"""The pair kernels' square root (one Newton-Raphson step on the hardware
estimate, Markstein's method) is the IEEE round-to-nearest one on every
float in [2^-60, FLT_MAX]: checked against CUDA's __fsqrt_rn on the device,
exhaustively."""
import pytest

from mars_md_b200.engine import Context

pytestmark = pytest.mark.gpu


def test_sqrt_matches_cuda_intrinsic_exhaustively():
    ctx = Context(1024)
    try:
        assert ctx.selftest_sqrt() == 0
    finally:
        ctx.close()
