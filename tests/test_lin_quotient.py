"""The LINEAR stencils' interpolation fraction t = a / b is formed from a table of correctly
rounded reciprocal spans y = RN(1/b) by Markstein's correction step (q0 = RN(a y), r = a - b q0
by one FMA, q = RN(q0 + r y); csrc/advect.cuh lin_quotient).  This checks that step against the
IEEE quotient on the host (same IEEE-754 binary64 / binary32 arithmetic and fused multiply-add as
the device), bit for bit: stencil-shaped cases (a point inside or just outside its bracket on
uniform and irregular lines, spans whose significands end in long runs of ones, spans over 30
binades) and random operands over 120 binades, in double and in float; and that the table the
kernels read holds those correctly rounded reciprocals.  No GPU needed."""
import os
import shutil
import subprocess

import pytest

SRC = r'''
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
static uint64_t s = 88172645463325252ull;
static uint64_t rnd(void) { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return s; }
static double u01(void) { return (rnd() >> 11) * (1.0 / 9007199254740992.0); }
static double qd(double a, double b, double y) { double q0 = a * y; double r = fma(-b, q0, a); return fma(r, y, q0); }
static float qf(float a, float b, float y) { float q0 = a * y; float r = fmaf(-b, q0, a); return fmaf(r, y, q0); }
static double rd(int emax) {
  uint64_t m = rnd() & 0x000fffffffffffffull; int e = 1023 + (int)(rnd() % (2 * emax + 1)) - emax;
  uint64_t v = ((uint64_t)e << 52) | m; if (rnd() & 1) v |= 1ull << 63; double d; memcpy(&d, &v, 8); return d;
}
int main(int argc, char **argv) {
  long n = atol(argv[1]), bad = 0, badf = 0, cnt = 0;
  for (long i = 0; i < n; i++) {
    double x0, x1, x;
    switch (i % 5) {
      case 0: x0 = u01() * 10 - 5; x1 = x0 + 1e-3 + u01(); x = x0 + (u01() * 1.2 - 0.1) * (x1 - x0); break;
      case 1: { double L = 6.283185307179586; int m = 1 + (int)(rnd() % 1024); double dx = L / m; int k = (int)(rnd() % m);
                x0 = (k + 0.5) * dx; x1 = (k + 1.5) * dx; x = x0 + u01() * dx; break; }
      case 2: { uint64_t bb = 0x3ff0000000000000ull | (rnd() & 0x000fffffffffffffull) | 0x000ffffffff00000ull; double b; memcpy(&b, &bb, 8);
                x0 = u01(); x1 = x0 + b; x = x0 + u01() * b; break; }
      case 3: x0 = u01() * 100; x1 = x0 + ldexp(1.0 + u01(), -(int)(rnd() % 30)); x = x0 + (u01() * 1.2 - 0.1) * (x1 - x0); break;
      default: x0 = 0.0; x = rd(60); x1 = rd(60); if (x1 < 0) x1 = -x1; break;
    }
    double b = x1 - x0, a = x - x0;
    if (b == 0) continue;
    cnt++;
    if (qd(a, b, 1.0 / b) != a / b) bad++;
    float af = (float)a, bf = (float)b;
    if (bf != 0.0f && isfinite(af / bf) && qf(af, bf, 1.0f / bf) != af / bf) badf++;
  }
  printf("%ld %ld %ld\n", cnt, bad, badf);
  return 0;
}
'''


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_markstein_quotient_equals_ieee_division(tmp_path):
    c, exe = tmp_path / "lq.c", tmp_path / "lq"
    c.write_text(SRC)
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", str(exe), str(c), "-lm"], check=True)
    out = subprocess.run([str(exe), "20000000"], check=True, capture_output=True, text=True).stdout.split()
    cnt, bad, badf = int(out[0]), int(out[1]), int(out[2])
    assert cnt > 19_000_000
    assert bad == 0 and badf == 0, out


HOST_SRC = r'''
#include <cstdio>
#include <vector>
#include "grid.h"
int main() {
  std::vector<double> l;
  std::vector<float> lf;
  double x = -3.0;
  unsigned long long s = 12345;
  for (int i = 0; i < 2000; i++) {
    s = s * 6364136223846793005ull + 1442695040888963407ull;
    x += 1e-3 + (double)(s >> 11) / 9007199254740992.0;
    l.push_back(x);
    lf.push_back((float)x);
  }
  l.push_back(x);  // a repeated line: zero span
  lf.push_back((float)x);
  const std::vector<double> r = cfd2lcs::reciprocal_spans(l);
  const std::vector<float> rf = cfd2lcs::reciprocal_spans(lf);
  for (size_t i = 0; i < l.size(); i++) printf("%a %a %a %a\n", l[i], r[i], (double)lf[i], (double)rf[i]);
  return 0;
}
'''


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_reciprocal_span_table_is_correctly_rounded(tmp_path):
    """The table the kernels read (csrc/grid.h reciprocal_spans): RN(1 / (l[i+1] - l[i])) in the
    table's own type, 0 for a zero span and at the last index."""
    import numpy as np
    here = os.path.dirname(os.path.abspath(__file__))
    csrc = os.path.join(os.path.dirname(here), "libcfd2lcs_b200", "csrc")
    c, exe = tmp_path / "rs.cpp", tmp_path / "rs"
    c.write_text(HOST_SRC)
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", csrc, "-o", str(exe), str(c)], check=True)
    rows = [ln.split() for ln in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines()]
    l = np.array([float.fromhex(r[0]) for r in rows])
    r = np.array([float.fromhex(r[1]) for r in rows])
    lf = np.array([float.fromhex(r[2]) for r in rows], dtype=np.float32)
    rf = np.array([float.fromhex(r[3]) for r in rows], dtype=np.float32)
    span = l[1:] - l[:-1]
    want = np.where(span != 0, 1.0 / np.where(span != 0, span, 1.0), 0.0)
    assert np.array_equal(r[:-1], want) and r[-1] == 0.0
    spanf = (lf[1:] - lf[:-1]).astype(np.float32)
    wantf = np.where(spanf != 0, np.float32(1) / np.where(spanf != 0, spanf, np.float32(1)), np.float32(0)).astype(np.float32)
    assert np.array_equal(rf[:-1], wantf) and rf[-1] == 0.0
    assert r[-2] == 0.0 and rf[-2] == 0.0  # the repeated line
