"""The Fortran half of the drop-in boundary: the gfortran-mangled entry points (cfd2lcs_init_,
cfd2lcs_diagnostic_init_, cfd2lcs_update_, cfd2lcs_set_option_, cfd2lcs_set_param_,
cfd2lcs_finalize_) called with gfortran's conventions -- scalars by reference, CHARACTER
arguments blank-padded without a terminating NUL plus a hidden trailing size_t length -- from a
compiled C driver (tests/c_driver/fortran_abi_driver.c; no Fortran compiler is installed).  On
the GPU the run through those symbols must give the same handle and bitwise the same FTLE as
the same run through the cfd2lcs_*_c entry points; without a GPU both paths latch the CUDA
error the same way."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import libcfd2lcs_b200 as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lib = L.library_path("dp")
    if not os.path.exists(lib):
        L.build(("dp",))
    exe = str(tmp_path / "fortran_abi_driver")
    cmd = [cc, "-O2", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "include", "mpistub"),
           os.path.join(ROOT, "tests", "c_driver", "fortran_abi_driver.c"), "-o", exe, "-L", os.path.dirname(lib),
           f"-l:{os.path.basename(lib)}", f"-Wl,-rpath,{os.path.dirname(lib)}", "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def _run(exe, mode, out):
    env = dict(os.environ, CFD2LCS_B200_QUIET="1")
    r = subprocess.run([exe, mode, str(out)], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout.strip().splitlines()[-1]


def test_fortran_symbols_latch_like_c_without_gpu(tmp_path):
    from tests.conftest import gpu_available
    exe = _build(tmp_path)
    if gpu_available():
        pytest.skip("a GPU is present (the run is covered by the gpu test)")
    a = _run(exe, "fortran", tmp_path / "f.bin")
    b = _run(exe, "c", tmp_path / "c.bin")
    assert a.startswith("error") and "CUDA" in a, a
    assert a == b


@pytest.mark.gpu
def test_fortran_symbols_match_c_entry_points(tmp_path):
    exe = _build(tmp_path)
    a = _run(exe, "fortran", tmp_path / "f.bin")
    b = _run(exe, "c", tmp_path / "c.bin")
    assert a.startswith("ok") and a == b, (a, b)
    fa = np.fromfile(tmp_path / "f.bin", dtype=np.float64)
    fb = np.fromfile(tmp_path / "c.bin", dtype=np.float64)
    assert fa.size == 14 ** 3 and np.all(np.isfinite(fa))
    assert np.array_equal(fa, fb)
    assert float(np.max(np.abs(fa))) > 0.0
