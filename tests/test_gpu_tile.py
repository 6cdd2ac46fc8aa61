"""The subcycle kernels that stage their taps in shared memory -- backward cubic (k_sl_tile),
backward LINEAR (k_sl_march_lin, planes marching along z, where the fields have tensor maps;
else k_sl_tile_lin) and forward cubic (k_fwd_tile, one block per 16 x 4 x 4-cell
sort tile) -- against the gathering kernels they replace (k_sl_subcycle, k_fwd_subcycle,
selected with CFD2LCS_B200_SL_TILE=0 at cfd2lcs_init): both contract the same taps in the same
order, so flow maps and FTLE must be bitwise equal.  Grids of 38^3 leave partial tiles in x (38 = 32 + 6), y and z (38 = 9 x 4 + 2);
the small walled / mixed-boundary cases clip the staged box at the padded array's edges.
The oracle parity of the same path is in test_gpu_parity.py and test_golden_configs.py."""
import os

import numpy as np
import pytest

from tests import scenarios as SC

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu_dp():
    import libcfd2lcs_b200 as L
    return L.Cfd2lcs("dp")


@pytest.fixture(scope="module")
def gpu_sp():
    import libcfd2lcs_b200 as L
    return L.Cfd2lcs("sp")


def _run(gpu, case, integrator, staged, n=None, steps=None, mixed=False, dirs=(SC.FTLE_BKWD,), interp=3, env=None):
    # 2 also stages the LINEAR backward kernel (off by default: slower than its gathering form)
    extra = dict(env or {}, CFD2LCS_B200_SL_TILE="2" if staged else "0")
    os.environ.update(extra)
    try:
        gpu.reset()
        if mixed:
            gpu.set_option("MIXED_PRECISION", 1)
        _, hs = SC.run(gpu, case, dirs, integrator, interp, n=n, steps=steps)
    finally:
        for k in extra:
            os.environ.pop(k, None)
    err, msg = gpu.error()
    assert err == 0, msg
    return [gpu.flowmap(h) for h in hs], [gpu.ftle(h) for h in hs], gpu.counters(), gpu.staged_launches()


def _same(gpu, case, integrator, **kw):
    fa, ta, ca, sa = _run(gpu, case, integrator, True, **kw)
    fb, tb, cb, sb = _run(gpu, case, integrator, False, **kw)
    key = "fwd" if kw.get("dirs") == (SC.FTLE_FWD,) else "sl"
    assert sa[key] > 0, "the staged kernel did not run"
    assert sb["sl"] == 0 and sb["fwd"] == 0
    assert ca["integrations_bkwd"] == cb["integrations_bkwd"] and ca["ftle_frames"] == cb["ftle_frames"]
    for x, y in zip(fa, fb):
        assert np.array_equal(x, y), f"flow maps differ: max {np.max(np.abs(x - y)):.3e}"
    for x, y in zip(ta, tb):
        assert np.array_equal(x, y), f"FTLE differs: max {np.max(np.abs(x - y)):.3e}"


@pytest.mark.parametrize("integrator", [0, 2, 3, 4])
def test_staged_abc_partial_tiles(gpu_dp, integrator):
    _same(gpu_dp, "abc", integrator, n=38, steps=14)


def test_staged_abc_unsteady_mixed_precision(gpu_dp):
    _same(gpu_dp, "abc_unsteady", 3, n=38, mixed=True)


@pytest.mark.parametrize("case", ["mixed_bc", "turb"])
def test_staged_small_and_walled(gpu_dp, case):
    _same(gpu_dp, case, 3)


def test_staged_single_precision(gpu_sp):
    _same(gpu_sp, "abc", 3, n=38, steps=14)


@pytest.mark.parametrize("integrator", [0, 2, 3, 4])
def test_staged_linear_abc_partial_tiles(gpu_dp, integrator):
    _same(gpu_dp, "abc", integrator, n=38, steps=14, interp=1)


def test_staged_linear_unsteady_mixed_precision(gpu_dp):
    _same(gpu_dp, "abc_unsteady", 2, n=38, mixed=True, interp=1)


@pytest.mark.parametrize("case", ["mixed_bc", "turb", "channel"])
def test_staged_linear_small_and_walled(gpu_dp, case):
    _same(gpu_dp, case, 2, interp=1)


@pytest.mark.parametrize("kc", ["1", "3", "7", "64"])
def test_staged_linear_march_runs(gpu_dp, kc):
    """k_sl_march_lin with column runs of 1, 3, 7 and all planes (38 = 5 x 7 + 3 leaves a
    partial run; a run of 1 plane issues no copy after its prologue): bitwise the gathering
    kernel, and the marching kernel is the one that ran."""
    env = {"CFD2LCS_B200_SL_MARCH_KC": kc}
    _same(gpu_dp, "abc", 3, n=38, steps=10, interp=1, env=env)
    _, _, _, sa = _run(gpu_dp, "abc", 3, True, n=38, steps=10, interp=1, env=env)
    assert sa["sl_march"] == sa["sl"] > 0


def test_staged_linear_boxes_without_march(gpu_dp):
    """CFD2LCS_B200_SL_MARCH=0 keeps the 32 x 4 x 4 boxes of k_sl_tile_lin: the same bits."""
    env = {"CFD2LCS_B200_SL_MARCH": "0"}
    _same(gpu_dp, "abc", 2, n=38, steps=10, interp=1, env=env)
    _, _, _, sa = _run(gpu_dp, "abc", 2, True, n=38, steps=10, interp=1, env=env)
    assert sa["sl_march"] == 0 and sa["sl"] > 0


def test_staged_linear_march_walled_channel(gpu_dp):
    """A walled channel (10 x 8 x 6, rows of 12 FP64 values: tensor maps exist): the marching
    kernel with boundary flags, runs of 4 planes."""
    env = {"CFD2LCS_B200_SL_MARCH_KC": "4"}
    _same(gpu_dp, "channel", 3, interp=1, env=env)
    _, _, _, sa = _run(gpu_dp, "channel", 3, True, interp=1, env=env)
    assert sa["sl_march"] == sa["sl"] > 0


def test_staged_linear_single_precision(gpu_sp):
    _same(gpu_sp, "turb", 3, n=20, interp=1)


@pytest.mark.parametrize("integrator", [0, 2, 3, 4])
def test_staged_forward_abc_partial_tiles(gpu_dp, integrator):
    _same(gpu_dp, "abc", integrator, n=38, steps=14, dirs=(SC.FTLE_FWD,))


def test_staged_forward_unsteady_mixed_precision(gpu_dp):
    _same(gpu_dp, "abc_unsteady", 3, n=38, mixed=True, dirs=(SC.FTLE_FWD,))


@pytest.mark.parametrize("case", ["mixed_bc", "turb"])
def test_staged_forward_small_and_walled(gpu_dp, case):
    _same(gpu_dp, case, 3, dirs=(SC.FTLE_FWD,))


def test_staged_forward_single_precision(gpu_sp):
    _same(gpu_sp, "abc", 3, n=38, steps=14, dirs=(SC.FTLE_FWD,))


def test_staged_both_directions(gpu_dp):
    """Forward and backward sets of one run (the benchmark's configuration)."""
    fa, ta, _, sa = _run(gpu_dp, "abc", 3, True, n=38, steps=14, dirs=(SC.FTLE_FWD, SC.FTLE_BKWD))
    fb, tb, _, _ = _run(gpu_dp, "abc", 3, False, n=38, steps=14, dirs=(SC.FTLE_FWD, SC.FTLE_BKWD))
    assert sa["sl"] > 0 and sa["fwd"] > 0
    for x, y in zip(fa + ta, fb + tb):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("dirs", [(SC.FTLE_BKWD,), (SC.FTLE_FWD,)])
def test_staged_row_copies(gpu_dp, dirs):
    """The boxes copied row by row (CFD2LCS_B200_TMA_TENSOR=0) instead of one tensor-map box per
    component: the same bits."""
    _same(gpu_dp, "abc", 3, n=38, steps=14, dirs=dirs, env={"CFD2LCS_B200_TMA_TENSOR": "0"})


@pytest.mark.parametrize("dirs", [(SC.FTLE_BKWD,), (SC.FTLE_FWD,)])
def test_staged_odd_pitch(gpu_dp, dirs):
    """37^3: a padded row of 39 FP64 values is not a multiple of 16 bytes, so no tensor map
    exists and the rows are copied with their per-row alignment shifts."""
    _same(gpu_dp, "abc", 3, n=37, steps=14, dirs=dirs)


def test_tuner_decides_and_keeps_bits(gpu_dp):
    """The default mode times both forms of each kernel on the first launches and keeps the
    faster: it reaches a choice for the backward and the forward kernel, and the run is bitwise
    the gathering-only run whichever it chose."""
    os.environ["CFD2LCS_B200_SL_TILE"] = "1"
    try:
        gpu_dp.reset()
        _, hs = SC.run(gpu_dp, "abc", (SC.FTLE_FWD, SC.FTLE_BKWD), 3, 3, n=38, steps=14)
    finally:
        os.environ.pop("CFD2LCS_B200_SL_TILE", None)
    err, msg = gpu_dp.error()
    assert err == 0, msg
    tu = gpu_dp.tuning()
    out = [gpu_dp.flowmap(h) for h in hs] + [gpu_dp.ftle(h) for h in hs]
    assert tu["bkwd"] in (0, 1) and tu["fwd"] in (0, 1), tu
    assert min(tu["bkwd_ms"]) > 0 and min(tu["fwd_ms"]) > 0, tu
    fb, tb, _, _ = _run(gpu_dp, "abc", 3, False, n=38, steps=14, dirs=(SC.FTLE_FWD, SC.FTLE_BKWD))
    for x, y in zip(out, fb + tb):
        assert np.array_equal(x, y)
