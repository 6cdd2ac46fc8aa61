"""Output files (write_lcs, src/io_nohdf5_m.f90:47-332): the Fortran ES editing of the values,
the file names, header and BLOCK layout of the oracle's restatement (CPU), and the library's
files against the oracle's (GPU)."""
import ctypes as C
import math
import os

import numpy as np
import pytest

from tests import workloads as W
from tests import scenarios as SC


@pytest.fixture(scope="module")
def gpu_dp():
    import libcfd2lcs_b200 as L
    return L.Cfd2lcs("dp")


def _fmt(v, w=14, d=6):
    import libcfd2lcs_b200 as L
    lib = L.load("dp")
    lib.cfd2lcs_b200_format_es.argtypes = [C.c_double, C.c_int, C.c_int, C.c_char_p]
    buf = C.create_string_buffer(64)
    lib.cfd2lcs_b200_format_es(v, w, d, buf)
    return buf.value.decode()


# ESw.d editing by the Fortran rules: one digit before the point, d after (rounded), E+xx
# for two-digit exponents, +xxx (no E) for three; right-justified; gfortran's NaN / Infinity
ES_KATS = [
    (1.0, 14, 6, "  1.000000E+00"),
    (-0.5, 14, 6, " -5.000000E-01"),
    (0.0, 14, 6, "  0.000000E+00"),
    (123456789.0, 14, 6, "  1.234568E+08"),
    (0.1, 14, 6, "  1.000000E-01"),
    (9.9999996, 14, 6, "  1.000000E+01"),
    (-1.2345674e-7, 14, 6, " -1.234567E-07"),
    (1e-300, 14, 6, "  1.000000-300"),
    (-2.5e150, 14, 6, " -2.500000+150"),
    (float("nan"), 14, 6, "           NaN"),
    (float("inf"), 14, 6, "      Infinity"),
    (float("-inf"), 14, 6, "     -Infinity"),
    (1.0, 18, 4, "        1.0000E+00"),
    (15.0, 18, 4, "        1.5000E+01"),
    (0.85, 18, 4, "        8.5000E-01"),
]


@pytest.mark.parametrize("v,w,d,expect", ES_KATS)
def test_es_editing(v, w, d, expect):
    assert _fmt(v, w, d) == expect


def _expected_frames(prm, directions):
    """(label, index) of every write_lcs file: a frame where int(t_np1/h) /= int(t_n/h)
    (src/cfd2lcs.f90:147), index nint(t/h), minus nint(T/h) for FTLE_FWD (io_nohdf5_m.f90:66-71)."""
    out = []
    t_prev = None
    for k in range(prm["steps"]):
        t = W.time_at(k, prm["dt"])
        if t_prev is not None and int(t / prm["h"]) != int(t_prev / prm["h"]):
            for d in directions:
                f = int(math.floor(t / prm["h"] + 0.5))
                if d == SC.FTLE_FWD:
                    f -= int(math.floor(prm["T"] / prm["h"] + 0.5))
                idx = f"{f:010d}" if 1000 <= f <= 9999 else str(f)
                out.append((f"d{d}", idx, t))
        t_prev = t
    return out


def _run(api, case, integrator, interp, options, directions=(SC.FTLE_BKWD, SC.FTLE_FWD)):
    g, vel, prm = SC.make_case(case)
    api.reset()
    api.init(g.n, g.x, g.y, g.z, g.flag)
    for d in directions:
        api.diagnostic_init(d, 0, prm["T"], prm["h"], f"d{d}")
    api.set_option("INTEGRATOR", integrator)
    api.set_option("INTERPOLATOR", interp)
    for k, v in options.items():
        api.set_option(k, v)
    for k in range(prm["steps"]):
        t = W.time_at(k, prm["dt"])
        api.update(*vel(t), t)
    return g, prm


def _parse(path):
    with open(path) as f:
        lines = f.read().split("\n")
    assert lines[-1] == ""
    lines = lines[:-1]
    k = lines.index("ZONETYPE = Ordered, DATAPACKING = BLOCK")
    return lines[: k + 1], lines[k + 1:]


def test_oracle_writer_layout(oracle_dp, tmp_path):
    """The oracle's write_lcs restatement against the reference's layout rules."""
    opts = {"WRITE_LCS": 1, "VELOCITY_INVARIANTS": 1, "WRITE_BCFLAG": 1}
    oracle_dp.set_output_dir(str(tmp_path))
    try:
        g, prm = _run(oracle_dp, "abc_unsteady", 2, 1, opts)
        assert oracle_dp.error() == 0, oracle_dp.error_msg()
    finally:
        oracle_dp.set_output_dir("")
    frames = _expected_frames(prm, (SC.FTLE_BKWD, SC.FTLE_FWD))
    assert sorted(os.listdir(tmp_path)) == sorted(f"{lab}_{idx}.dat" for lab, idx, _ in frames)
    npts = int(np.prod(g.n))
    for lab, idx, t in frames:
        head, data = _parse(tmp_path / f"{lab}_{idx}.dat")
        names = ["X", "Y", "Z", "FM-X", "FM-Y", "FM-Z", "U-X", "U-Y", "U-Z", "FLAG", "Q", "C", "D", "H", "L2", "FTLE"]
        assert head[:2] == [f'TITLE = "{lab}-FTLE"', "VARIABLES ="]
        assert head[2:2 + len(names)] == [f'"{v}"' for v in names]
        assert head[2 + len(names):] == ["ZONE", f'T = "{lab}-FTLE"', f"STRANDID = 0000000001, SOLUTIONTIME = {_fmt(t, 18, 4)}",
                                          f"I = {g.n[0]:010d} J = {g.n[1]:010d} K = {g.n[2]:010d}",
                                          "ZONETYPE = Ordered, DATAPACKING = BLOCK"]
        per_block = (npts + 9) // 10
        assert len(data) == len(names) * per_block
        for b in range(len(names)):
            blk = data[b * per_block:(b + 1) * per_block]
            assert all(len(s) == 140 for s in blk[:-1]) and len(blk[-1]) == 14 * (npts - 10 * (per_block - 1))
        xs = np.array([float(s[14 * q:14 * q + 14]) for s in data[:per_block] for q in range(len(s) // 14)])
        np.testing.assert_allclose(xs, g.x.ravel(order="F"), rtol=1e-6)
        fl = np.array([float(s[14 * q:14 * q + 14]) for s in data[9 * per_block:10 * per_block] for q in range(len(s) // 14)])
        assert np.array_equal(fl, g.flag.ravel(order="F").astype(float))


def _values(lines):
    return [s[14 * q:14 * q + 14] for s in lines for q in range(len(s) // 14)]


def _compare_files(pa, pb, rtol, bitwise_blocks, flag_blocks=(), skip_blocks=()):
    """flag_blocks: 0/1/... indicator blocks (the invariants' Q, C, D, L2 flags), which may
    differ at a few nodes where the indicator sits at a rounding tie, as the invariants'
    parity test allows (max(2, n/500) nodes)."""
    ha, da = _parse(pa)
    hb, db = _parse(pb)
    assert ha == hb
    assert [len(s) for s in da] == [len(s) for s in db]
    va, vb = _values(da), _values(db)
    nb = len(ha) - 7
    per = len(va) // nb
    for b in range(nb):
        A, B = va[b * per:(b + 1) * per], vb[b * per:(b + 1) * per]
        if b in skip_blocks:
            continue
        if b in bitwise_blocks:
            assert A == B, b
            continue
        if b in flag_blocks:
            assert sum(x != y for x, y in zip(A, B)) <= max(2, len(A) // 500), b
            continue
        fa = np.array([float(s) for s in A])
        fb = np.array([float(s) for s in B])
        same = np.isnan(fa) == np.isnan(fb)
        assert np.all(same), b
        ok = np.isnan(fa) | np.isclose(fa, fb, rtol=rtol, atol=1e-9)
        assert np.all(ok), (b, np.max(np.abs(fa - fb)[~ok]))


@pytest.mark.gpu
@pytest.mark.parametrize("case,integrator,interp,opts", [
    ("abc_unsteady", 2, 1, {"VELOCITY_INVARIANTS": 1, "WRITE_BCFLAG": 1}),
    ("mixed_bc", 3, 3, {}),
    ("dg", 2, 1, {"WRITE_FLOWMAP": 0, "WRITE_VELOCITY": 0, "WRITE_LCS_ASYNC": 1}),
    ("curv_box", 2, 6, {"VELOCITY_INVARIANTS": 1}),  # non-rectilinear: node coordinates, not lines
])
def test_writer_matches_oracle(oracle_dp, gpu_dp, tmp_path, monkeypatch, case, integrator, interp, opts):
    """Same files, names and headers as the oracle's; grid and flag blocks identical text;
    the computed blocks equal to the 7 printed digits (the parity tolerance is far below the
    last printed digit, so only a rounding neighbour can differ)."""
    odir = tmp_path / "oracle"
    odir.mkdir()
    oracle_dp.set_output_dir(str(odir))
    try:
        _run(oracle_dp, case, integrator, interp, {"WRITE_LCS": 1, **{k: v for k, v in opts.items() if k != "WRITE_LCS_ASYNC"}})
        assert oracle_dp.error() == 0, oracle_dp.error_msg()
    finally:
        oracle_dp.set_output_dir("")
    gdir = tmp_path / "gpu"
    gdir.mkdir()
    monkeypatch.chdir(gdir)
    try:
        _run(gpu_dp, case, integrator, interp, {"WRITE_LCS": 1, **opts})
        assert gpu_dp.error()[0] == 0, gpu_dp.error()
    finally:
        gpu_dp.reset()  # finishes background files
    names = sorted(os.listdir(odir))
    assert names and names == sorted(os.listdir(gdir / "cfd2lcs_output"))
    bitwise = {0, 1, 2}
    if opts.get("WRITE_BCFLAG"):
        bitwise.add(9)
    for nm in names:
        _compare_files(odir / nm, gdir / "cfd2lcs_output" / nm, rtol=2e-6, bitwise_blocks=bitwise)
