"""The FP64 FMA micro-benchmark the bench reports the B-spline kernels' arithmetic against
(cfd2lcs_b200_fp64_fma_rate): it runs through the C ABI and returns a plausible B200 rate."""
import pytest

pytestmark = pytest.mark.gpu


def test_fp64_fma_rate():
    import libcfd2lcs_b200 as L
    r = L.Cfd2lcs("dp").fp64_fma_tflops(iters=2048, reps=3)
    assert 5.0 < r < 200.0, r
