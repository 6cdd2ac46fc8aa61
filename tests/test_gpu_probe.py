"""The FP64 FMA micro-benchmark the bench reports the B-spline kernels' arithmetic against
(libcfd2lcs_b200_fp64probe.so, a measurement library kept out of the drop-in): it runs and
returns a plausible B200 rate."""
import pytest

pytestmark = pytest.mark.gpu


def test_fp64_fma_rate():
    import bench
    r = bench.fp64_fma_tflops(iters=2048, reps=3)
    assert 5.0 < r < 200.0, r
