"""The batched form (cfd2lcs_batch_*): every instance of a batch must give exactly the result
of the same instance run alone through the reference interface (the same kernels on the same
inputs), for mixed grid kinds, sizes, directions and horizons advanced by one call."""
import numpy as np
import pytest

from tests import workloads as W
from tests import scenarios as SC

pytestmark = pytest.mark.gpu

# (case, grid n, lcs type, T, h, integrator, interpolator, mixed precision)
INSTANCES = [
    ("dg", 64, SC.FTLE_BKWD, 1.5, 0.15, 2, 1, False),
    ("abc", 12, SC.FTLE_FWD, 0.6, 0.2, 2, 1, False),
    ("dg", 48, SC.FTLE_FWD, 1.0, 0.2, 3, 3, False),
    ("abc", 16, SC.FTLE_BKWD, 1.0, 0.25, 3, 3, False),
    ("turb", 12, SC.FTLE_BKWD, 0.2, 0.05, 2, 1, True),
    ("abc", 12, SC.FTLE_BKWD, 0.6, 0.2, 3, 6, False),
]
STEPS = 20


def _single(api, case, n, lcs_type, T, h, integ, interp, mixed):
    g, vel, prm = SC.make_case(case, n)
    api.reset()
    if mixed:
        api.set_option("MIXED_PRECISION", 1)
    api.init(g.n, g.x, g.y, g.z, g.flag)
    hd = api.diagnostic_init(lcs_type, 0, T, h, "x")
    api.set_option("INTEGRATOR", integ)
    api.set_option("INTERPOLATOR", interp)
    for k in range(STEPS):
        t = W.time_at(k, prm["dt"])
        api.update(*vel(t), t)
    assert api.error()[0] == 0, api.error()
    out = api.ftle(hd).copy(), api.flowmap(hd).copy(), api.counters()
    api.reset()
    return out


def test_batch_matches_single_instances():
    import torch

    import libcfd2lcs_b200 as L
    api = L.Cfd2lcs("dp")
    ref = [_single(api, *spec) for spec in INSTANCES]

    b = L.Batch("dp")
    b.reset()
    ids, hds, vels, dts = [], [], [], []
    for case, n, lcs_type, T, h, integ, interp, mixed in INSTANCES:
        g, vel, prm = SC.make_case(case, n)
        i = b.add(g.n, g.x, g.y, g.z, g.flag, integ, interp, 0.5, mixed)
        assert i >= 0, b.error()
        hds.append(b.diagnostic_init(i, lcs_type, T, h))
        ids.append(i)
        vels.append(vel)
        dts.append(prm["dt"])
    assert b.error()[0] == 0, b.error()
    for k in range(STEPS):
        fields = []
        for vel, dt in zip(vels, dts):
            u, v, w = vel(W.time_at(k, dt))
            fields.append([torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"), dtype=np.float64)).cuda() for a in (u, v, w)])
        rc = b.update_device(ids, [f[0].data_ptr() for f in fields], [f[1].data_ptr() for f in fields],
                             [f[2].data_ptr() for f in fields], [W.time_at(k, dt) for dt in dts])
        assert rc == 0, b.error()
        torch.cuda.synchronize()
    for q, (i, hd) in enumerate(zip(ids, hds)):
        f_ref, m_ref, c_ref = ref[q]
        np.testing.assert_array_equal(b.ftle(i, hd), f_ref)
        np.testing.assert_array_equal(b.flowmap(i, hd), m_ref)
        cb = b.counters(i)
        for key in ("integrations_fwd", "integrations_bkwd", "ftle_frames", "updates"):
            assert cb[key] == c_ref[key], (q, key)
    b.reset()


def test_batch_reports_errors():
    import libcfd2lcs_b200 as L
    b = L.Batch("dp")
    b.reset()
    g = W.abc_grid(8)
    assert b.add(g.n, g.x, g.y, g.z, g.flag, 9, 1) == -1
    err, msg = b.error()
    assert err == 1 and "integrator" in msg
    b.reset()
    assert b.error()[0] == 0
