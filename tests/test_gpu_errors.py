"""Failure detection on the GPU path, made on the host (nothing here faults, traps or hangs the
device): a non-finite velocity caught by the device error word, a velocity array of the wrong
size, an unknown option, an unknown interpolator.  Each latches the error as the reference's
CFD2LCS_ERROR does (src/cfd2lcs.f90:684-706): the call reports it, later calls do nothing, and
after a reset the same process runs a clean case on the same device."""
import ctypes as C

import numpy as np
import pytest

from tests import workloads as W
from tests import scenarios as SC

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    import libcfd2lcs_b200 as L
    return L.Cfd2lcs("dp")


def _start(api, case="abc_unsteady"):
    g, vel, prm = SC.make_case(case)
    api.reset()
    api.init(g.n, g.x, g.y, g.z, g.flag)
    h = api.diagnostic_init(SC.FTLE_BKWD, 0, prm["T"], prm["h"], "b")
    assert api.error()[0] == 0, api.error()
    return g, vel, prm, h


def _clean_run_after(api):
    """The device context stays usable: a reset and a normal run succeed."""
    g, vel, prm, h = _start(api, "dg")
    for k in range(prm["steps"]):
        t = W.time_at(k, prm["dt"])
        api.update(*vel(t), t)
    assert api.error()[0] == 0, api.error()
    assert np.all(np.isfinite(api.ftle(h)))
    api.reset()


def test_non_finite_velocity_latches(api):
    g, vel, prm, h = _start(api)
    for k in range(3):
        t = W.time_at(k, prm["dt"])
        u, v, w = vel(t)
        if k == 2:
            u = np.array(u, copy=True)
            u[3, 4, 5] = np.nan
        api.update(u, v, w, t)
    err, msg = api.error()
    assert err != 0 and "non-finite" in msg, msg
    c = api.counters()["updates"]
    t = W.time_at(3, prm["dt"])
    api.update(*vel(t), t)  # latched: nothing runs
    assert api.counters()["updates"] == c
    _clean_run_after(api)


def test_wrong_array_size_latches(api):
    g, vel, prm, h = _start(api)
    u, v, w = (np.asfortranarray(a, dtype=np.float64).ravel(order="F") for a in vel(0.0))
    bad = np.array([g.n[0] - 1, g.n[1], g.n[2]], dtype=np.int32)
    api.lib.cfd2lcs_update_c(bad.ctypes.data_as(C.c_void_p), u.ctypes.data_as(C.c_void_p), v.ctypes.data_as(C.c_void_p),
                             w.ctypes.data_as(C.c_void_p), C.c_double(0.0))
    err, msg = api.error()
    assert err != 0 and "dimension" in msg, msg
    _clean_run_after(api)


@pytest.mark.parametrize("opt,val,text", [("NOT_AN_OPTION", 1, "option"), ("INTERPOLATOR", 4, "option")])
def test_bad_option_latches(api, opt, val, text):
    _start(api)
    api.set_option(opt, val)
    err, msg = api.error()
    assert err != 0 and text in msg, msg
    _clean_run_after(api)


def test_info_table(api, capfd, monkeypatch):
    """cfd2lcs_info's table (src/cfd2lcs.f90:708-810) after each update but the first, when
    CFD2LCS_B200_INFO is set: the reference's rows, and this step's backward integrations equal
    to the library's counter."""
    monkeypatch.setenv("CFD2LCS_B200_INFO", "1")
    g, vel, prm, h = _start(api)
    capfd.readouterr()
    counts = []
    for k in range(4):
        t = W.time_at(k, prm["dt"])
        c0 = api.counters()["integrations_bkwd"]
        api.update(*vel(t), t)
        counts.append(api.counters()["integrations_bkwd"] - c0)
    out = capfd.readouterr().out
    monkeypatch.delenv("CFD2LCS_B200_INFO")
    api.reset()
    tables = out.split("-----libcfd2lcs CPU overhead (NOT synchronized, rank 0 only)------")[1:]
    assert len(tables) == 3, out
    for label in ("|Application, Total:    |", "|cfd2lcs, BKWD Advect:  |", "|cfd2lcs, LCS:          |",
                  "| PARTICLE INTEGRATIONS |", "|Backward (cumulative): |"):
        assert label in tables[-1]
    line = [ln for ln in tables[-1].splitlines() if ln.startswith("|Backward (this step):  |")][0]
    assert counts[-1] > 0
    assert abs(float(line.split("|")[2]) - counts[-1]) <= 1e-4 * counts[-1]  # ES18.4: 4 significant digits
