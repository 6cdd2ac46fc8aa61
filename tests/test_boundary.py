"""The drop-in boundary: the C-ABI library builds, loads, exports every symbol the headers
declare, and has no CPU fallback (its compute entry points latch an error without a GPU)."""
import ctypes
import os
import re

import pytest

import libcfd2lcs_b200 as L
from tests import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return set(re.findall(r"\b(cfd2lcs_[a-z_0-9]+)\s*\(", src))


@pytest.mark.parametrize("prec", ["dp", "sp"])
def test_exports_every_declared_symbol(prec):
    path = L.library_path(prec)
    if not os.path.exists(path):
        L.build((prec,))
    lib = ctypes.CDLL(path)
    hdr = "cfd2lcs_inc_dp.h" if prec == "dp" else "cfd2lcs_inc_sp.h"
    names = _declared(hdr) | _declared("cfd2lcs_b200.h") | set(L.EXPORTED_SYMBOLS)
    assert len(names) >= 20
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_headers_match_reference_constants():
    src = open(os.path.join(ROOT, "include", "cfd2lcs_inc_dp.h")).read()
    vals = dict(re.findall(r"#define\s+(\w+)\s+(-?\d+)", src))
    expect = dict(LCS_INTERNAL=0, LCS_INFLOW=1, LCS_OUTFLOW=2, LCS_WALL=3, LCS_SLIP=4, LCS_2D=5, LCS_MASK=6, FTLE_FWD=0,
                  FTLE_BKWD=1, LP_TRACER=2, EULER=0, TRAPEZOIDAL=1, RK2=2, RK3=3, RK4=4, NEAREST_NBR=0, LINEAR=1, QUADRATIC=2,
                  CUBIC=3, TSE=5, TSE_LIMIT=6, LCS_FALSE=0, LCS_TRUE=1, LCS_NAMELEN=128)
    for k, v in expect.items():
        assert int(vals[k]) == v, k
    assert "typedef double lcsdata_t" in src
    assert "typedef float lcsdata_t" in open(os.path.join(ROOT, "include", "cfd2lcs_inc_sp.h")).read()


def test_no_cpu_fallback_without_gpu():
    from tests.conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    api = L.Cfd2lcs("dp")
    api.reset()
    g = W.abc_grid(4)
    api.init(g.n, g.x, g.y, g.z, g.flag)
    err, msg = api.error()
    assert err == 1 and "CUDA" in msg
    api.reset()
