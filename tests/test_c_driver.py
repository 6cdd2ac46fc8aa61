"""A C solver compiled against the drop-in headers (include/cfd2lcs_inc_dp.h, the MPI stub and
the extensions) and linked to libcfd2lcs_b200_dp.so, as a CFD code links the reference."""
import os
import shutil
import subprocess

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
    exe = str(tmp_path / "dg_driver")
    cmd = [cc, "-O2", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "include", "mpistub"),
           os.path.join(ROOT, "tests", "c_driver", "dg_driver.c"), "-o", exe, "-L", os.path.dirname(lib), f"-l:{os.path.basename(lib)}",
           f"-Wl,-rpath,{os.path.dirname(lib)}", "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def _run(exe):
    env = dict(os.environ, CFD2LCS_B200_QUIET="1")
    r = subprocess.run([exe], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout.strip().splitlines()[-1]


def test_c_driver_compiles_and_latches_without_gpu(tmp_path):
    from tests.conftest import gpu_available
    exe = _build(tmp_path)
    if gpu_available():
        pytest.skip("a GPU is present (the run is covered by the gpu test)")
    out = _run(exe)
    assert out.startswith("error") and "CUDA" in out, out


@pytest.mark.gpu
def test_c_driver_runs_on_the_gpu(tmp_path):
    exe = _build(tmp_path)
    out = _run(exe)
    assert out.startswith("ok"), out
    assert 0.0 < float(out.split()[1]) < 10.0
