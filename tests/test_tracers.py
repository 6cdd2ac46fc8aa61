"""LP_TRACER diagnostics (init_lp_tracer, src/lp_m.f90:116-226; update_lp, src/lp_motion_m.f90:
15-54; lifetime and output, src/cfd2lcs.f90:225-231): the oracle's restatement against the
injection rule and a translation known answer (CPU), and the library against the oracle (GPU)."""
import os

import numpy as np
import pytest

from tests import workloads as W
from tests import scenarios as SC

LP_TRACER = 2


@pytest.fixture(scope="module")
def gpu_dp():
    import libcfd2lcs_b200 as L
    return L.Cfd2lcs("dp")


def _inject(api, g, centre, radius):
    for name, v in zip(("TRACER_INJECT_X", "TRACER_INJECT_Y", "TRACER_INJECT_Z"), centre):
        api.set_param(name, v)
    api.set_param("TRACER_INJECT_RADIUS", radius)


def test_oracle_injection_rule(oracle_dp):
    """One tracer per node with |x - c| <= r, in node order; none inside: handle -1 and the
    number is used up (the next diagnostic gets the one after)."""
    g = W.abc_grid(12)
    oracle_dp.reset()
    oracle_dp.init(g.n, g.x, g.y, g.z, g.flag)
    assert oracle_dp.diagnostic_init(LP_TRACER, 0, 1.0, 0.5, "none") == -1  # default centre: huge
    c, r = (3.0, 2.5, 3.3), 1.1
    _inject(oracle_dp, g, c, r)
    h = oracle_dp.diagnostic_init(LP_TRACER, 0, 1.0, 0.5, "tr")
    assert h == 2
    X = np.stack([a.ravel(order="F") for a in (g.x, g.y, g.z)])
    inside = np.sqrt(((X - np.array(c)[:, None]) ** 2).sum(0)) <= r
    np.testing.assert_array_equal(oracle_dp.tracers(h), X[:, inside])
    assert oracle_dp.error() == 0


def test_oracle_translation_and_lifetime(oracle_dp):
    """Uniform velocity on a periodic cube: x(t) = x0 + U t wrapped into the domain; after the
    frame at which the lifetime exceeds T the tracers stop."""
    g = W.abc_grid(10)
    L = 2 * np.pi
    U = np.array([0.7, -0.4, 0.25])
    oracle_dp.reset()
    oracle_dp.init(g.n, g.x, g.y, g.z, g.flag)
    _inject(oracle_dp, g, (np.pi, np.pi, np.pi), 1.5)
    T, h, dt = 0.6, 0.2, 0.05
    hd = oracle_dp.diagnostic_init(LP_TRACER, 0, T, h, "tr")
    x0 = oracle_dp.tracers(hd).copy()
    vel = [np.full(g.x.shape, u) for u in U]
    stop, life, t_prev = None, 0.0, None
    for k in range(24):
        t = W.time_at(k, dt)
        oracle_dp.update(*vel, t)
        assert oracle_dp.counter("nsub_fwd") == 1
        xt = oracle_dp.tracers(hd)
        if stop is None:
            exp = x0 + U[:, None] * t
            d = (xt - exp + L / 2) % L - L / 2  # equal modulo the period
            assert np.max(np.abs(d)) < 1e-12
            if t_prev is not None:
                life = life + abs(t - t_prev)  # one subcycle per update here
                if int(t / h) != int(t_prev / h) and life > T:
                    stop = xt.copy()
        else:
            np.testing.assert_array_equal(xt, stop)
        t_prev = t
    assert stop is not None
    assert oracle_dp.error() == 0


def _run(api, case, integrator, interp, centre, radius, opts=None, steps=None):
    g, vel, prm = SC.make_case(case)
    api.reset()
    api.init(g.n, g.x, g.y, g.z, g.flag)
    _inject(api, g, centre, radius)
    hb = api.diagnostic_init(SC.FTLE_BKWD, 0, prm["T"], prm["h"], "b")
    ht = api.diagnostic_init(LP_TRACER, 0, prm["T"], prm["h"], "tr")
    api.set_option("INTEGRATOR", integrator)
    api.set_option("INTERPOLATOR", interp)
    for k, v in (opts or {}).items():
        api.set_option(k, v)
    for k in range(steps or prm["steps"]):
        t = W.time_at(k, prm["dt"])
        api.update(*vel(t), t)
    return g, hb, ht


CASES = [
    ("abc_unsteady", 2, 1, (2.0, 3.0, 4.0), 1.6),
    ("mixed_bc", 3, 3, (0.5, 0.5, 0.45), 0.35),
    ("dg", 4, 1, (1.0, 0.5, 0.0), 0.3),
    ("abc_unsteady", 3, 6, (2.0, 3.0, 4.0), 1.6),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case,res", [("abc_unsteady", 1), ("dg", 2)])
def test_tracers_on_refined_grid_match_oracle(oracle_dp, gpu_dp, case, res):
    """resolution /= 0: the refined lcs grid's nodes inside the sphere are injected and tracked
    to the solver grid (with the periodic wrap), then advected on the solver grid."""
    def run(api):
        g, vel, prm = SC.make_case(case)
        api.reset()
        api.init(g.n, g.x, g.y, g.z, g.flag)
        _inject(api, g, (2.0, 3.0, 4.0) if case == "abc_unsteady" else (1.0, 0.5, 0.0), 1.6 if case == "abc_unsteady" else 0.3)
        h = api.diagnostic_init(LP_TRACER, res, prm["T"], prm["h"], "tr")
        api.set_option("INTEGRATOR", 2)
        api.set_option("INTERPOLATOR", 1)
        for k in range(prm["steps"]):
            t = W.time_at(k, prm["dt"])
            api.update(*vel(t), t)
        return g, h
    g, ho = run(oracle_dp)
    assert oracle_dp.error() == 0, oracle_dp.error_msg()
    xo = oracle_dp.tracers(ho)
    try:
        _, hg = run(gpu_dp)
        assert gpu_dp.error()[0] == 0, gpu_dp.error()
        xg = gpu_dp.tracers(hg)
        assert xg.shape == xo.shape and xo.shape[1] > 0
        span = max(float(np.ptp(a)) for a in (g.x, g.y, g.z))
        np.testing.assert_allclose(xg, xo, rtol=0, atol=1e-12 * span)
    finally:
        gpu_dp.reset()


@pytest.mark.gpu
@pytest.mark.parametrize("case,integrator,interp,centre,radius", CASES)
def test_tracers_match_oracle(oracle_dp, gpu_dp, case, integrator, interp, centre, radius):
    g, hb, ht = _run(oracle_dp, case, integrator, interp, centre, radius)
    assert oracle_dp.error() == 0, oracle_dp.error_msg()
    xo = oracle_dp.tracers(ht)
    assert xo.shape[1] > 0
    try:
        _, hb2, ht2 = _run(gpu_dp, case, integrator, interp, centre, radius)
        assert (hb2, ht2) == (hb, ht)
        assert gpu_dp.error()[0] == 0, gpu_dp.error()
        xg = gpu_dp.tracers(ht2)
        span = max(float(np.ptp(a)) for a in (g.x, g.y, g.z))
        np.testing.assert_allclose(xg, xo, rtol=0, atol=1e-12 * span)
        assert gpu_dp.counters()["integrations_fwd"] == oracle_dp.counter("integrations_fwd")
    finally:
        gpu_dp.reset()


@pytest.mark.gpu
def test_tracer_files_match_oracle(oracle_dp, gpu_dp, tmp_path, monkeypatch):
    odir = tmp_path / "o"
    odir.mkdir()
    oracle_dp.set_output_dir(str(odir))
    try:
        _run(oracle_dp, "abc_unsteady", 2, 1, (2.0, 3.0, 4.0), 1.6, {"WRITE_LCS": 1})
        assert oracle_dp.error() == 0, oracle_dp.error_msg()
    finally:
        oracle_dp.set_output_dir("")
    gdir = tmp_path / "g"
    gdir.mkdir()
    monkeypatch.chdir(gdir)
    try:
        _run(gpu_dp, "abc_unsteady", 2, 1, (2.0, 3.0, 4.0), 1.6, {"WRITE_LCS": 1})
        assert gpu_dp.error()[0] == 0, gpu_dp.error()
    finally:
        gpu_dp.reset()
    names = sorted(n for n in os.listdir(odir) if n.startswith("tr_"))
    assert names and names == sorted(n for n in os.listdir(gdir / "cfd2lcs_output") if n.startswith("tr_"))
    for nm in names:
        ho, do = _parse_point(odir / nm)
        hg, dg = _parse_point(gdir / "cfd2lcs_output" / nm)
        assert ho == hg
        assert [len(s) for s in do] == [len(s) for s in dg] and all(len(s) == 42 for s in do)
        a = np.array([[float(s[14 * q:14 * q + 14]) for q in range(3)] for s in do])
        b = np.array([[float(s[14 * q:14 * q + 14]) for q in range(3)] for s in dg])
        np.testing.assert_allclose(a, b, rtol=2e-6, atol=1e-9)


def _parse_point(path):
    with open(path) as f:
        lines = f.read().split("\n")[:-1]
    k = lines.index("ZONETYPE = Ordered, DATAPACKING = POINT")
    return lines[: k + 1], lines[k + 1:]
