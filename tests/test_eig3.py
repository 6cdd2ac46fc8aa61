"""The closed-form largest eigenvalue of a symmetric 3x3 (libcfd2lcs_b200/csrc/eig3.h) that
the FTLE kernels use in place of the reference's per-point LAPACK DSYEV (src/lcs_m.f90:160-177),
and of the Jacobi iteration it falls back to where the two largest eigenvalues (nearly)
coincide, compiled for the host and checked against LAPACK (numpy.linalg.eigvalsh): random
Cauchy-Green-like tensors, near-degenerate spectra (two and three equal eigenvalues, rotated),
and wide ranges (largest over smallest eigenvalue up to 1e16, magnitudes 1e-150 to 1e150).
Bound: 1e-13 of the largest |eigenvalue| (the FTLE is log(sqrt(lambda))/T, so this is far below
the 1e-9 FTLE parity tolerance)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def eig3(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    exe = str(tmp_path_factory.mktemp("eig3") / "eig3_check")
    r = subprocess.run([cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "libcfd2lcs_b200", "csrc"),
                        os.path.join(ROOT, "tests", "c_driver", "eig3_check.cpp"), "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr

    def run(mats):
        rows = "\n".join(" ".join(repr(float(v)) for v in (m[0, 0], m[0, 1], m[0, 2], m[1, 1], m[1, 2], m[2, 2])) for m in mats)
        out = subprocess.run([exe], input=rows, capture_output=True, text=True, check=True).stdout.split()
        return np.array([float(v) for v in out]).reshape(-1, 2)

    return run


def _rot(rng):
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    return q


def _check(eig3, mats):
    got = eig3(mats)
    ref = np.array([np.linalg.eigvalsh(m)[-1] for m in mats])
    scale = np.array([np.max(np.abs(np.linalg.eigvalsh(m))) for m in mats])
    for col, name in ((0, "closed form"), (1, "Jacobi")):
        err = np.abs(got[:, col] - ref) / np.where(scale > 0, scale, 1.0)
        assert float(err.max()) <= 1e-13, (name, float(err.max()), mats[int(err.argmax())])


def test_random_cauchy_green(eig3):
    rng = np.random.default_rng(1)
    mats = []
    for _ in range(2000):
        G = rng.normal(size=(3, 3)) * 10.0 ** rng.uniform(-3, 3)
        mats.append(G.T @ G)
    _check(eig3, mats)


def test_near_degenerate(eig3):
    rng = np.random.default_rng(2)
    mats = []
    for _ in range(600):
        lam = rng.uniform(0.1, 10.0)
        for w in ([lam, lam, lam * (1 + 1e-9)], [lam * (1 - 1e-12), lam, lam], [0.0, lam, lam], [lam, lam, lam], [0.0, 0.0, lam]):
            R = _rot(rng)
            mats.append(R @ np.diag(w) @ R.T)
    _check(eig3, mats)


def test_wide_range(eig3):
    rng = np.random.default_rng(3)
    mats = []
    for _ in range(600):
        top = 10.0 ** rng.uniform(-150, 150)
        w = np.sort([top * 10.0 ** -rng.uniform(0, 16), top * 10.0 ** -rng.uniform(0, 16), top])
        R = _rot(rng)
        mats.append(R @ np.diag(w) @ R.T)
    _check(eig3, mats)


def test_zero_and_nan(eig3):
    z = np.zeros((3, 3))
    n = np.full((3, 3), np.nan)
    got = eig3([z, n])[:, 0]
    assert got[0] == 0.0 and np.isnan(got[1])
