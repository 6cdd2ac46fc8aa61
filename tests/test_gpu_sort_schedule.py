"""The forward particle sets' re-sort schedule: particles are advanced independently and read
back through the inverse slot map, so when they are re-sorted by cell changes only speed.  The
adaptive schedule of the gathering forward kernel (re-sort once the launch time lost since the
last sort reaches the sort's own time), a fixed interval of 2 subcycles and no re-sort at all
must give the same bits (LINEAR forward sets: the steady ABC flow, the unsteady double gyre with
slip walls, the mixed-boundary box)."""
import os

import numpy as np
import pytest

from tests import scenarios as SC

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu_dp():
    import libcfd2lcs_b200 as L
    return L.Cfd2lcs("dp")


def _run(gpu, case, every, n=None, steps=None):
    env = {} if every is None else {"CFD2LCS_B200_SORT_EVERY": str(every)}
    os.environ.update(env)
    try:
        gpu.reset()
        _, hs = SC.run(gpu, case, (SC.FTLE_FWD,), 2, 1, n=n, steps=steps)
    finally:
        for k in env:
            os.environ.pop(k, None)
    err, msg = gpu.error()
    assert err == 0, msg
    return [gpu.flowmap(h) for h in hs] + [gpu.ftle(h) for h in hs], gpu.counters()


@pytest.mark.parametrize("case,n,steps", [("abc", 24, 20), ("dg", 64, 40), ("mixed_bc", None, None)])
def test_sort_schedule_keeps_bits(gpu_dp, case, n, steps):
    ref, cref = _run(gpu_dp, case, 2, n, steps)
    for every in (None, 1000000, 5):
        out, c = _run(gpu_dp, case, every, n, steps)
        assert c["integrations_fwd"] == cref["integrations_fwd"]
        for a, b in zip(out, ref):
            assert np.array_equal(a, b), (case, every)
