"""Builds libcfd2lcs_b200_{dp,sp}.so in-tree with nvcc for sm_100a.

    python -m libcfd2lcs_b200.build            # both precisions
    python -m libcfd2lcs_b200.build dp         # one of them

The libraries link the CUDA runtime statically, so at run time they need only the
driver (libcuda).  No torch types cross the C ABI.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.environ.get("CFD2LCS_B200_BUILDDIR") or os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["engine.cu", "engine_mixed.cu", "adjoint.cu", "grid.cpp", "spline_host.cpp", "writer.cpp", "capi.cpp"]
# the FP64 FMA micro-benchmark bench.py reports the B-spline kernels against: a separate
# measurement library, not part of the drop-in
PROBE_SOURCE = "probe.cu"
HEADERS = ["grid.h", "engine.h", "engine_impl.cuh", "adjoint.h", "device_common.cuh", "advect.cuh", "spline.cuh", "kernels.cuh", "tile.cuh", "eig3.h", "spline_host.h", "writer.h"]


def lib_path(prec: str) -> str:
    return os.path.join(os.environ.get("CFD2LCS_B200_LIBDIR") or HERE, f"libcfd2lcs_b200_{prec}.so")


def probe_path() -> str:
    return os.path.join(os.environ.get("CFD2LCS_B200_LIBDIR") or HERE, "libcfd2lcs_b200_fp64probe.so")


def build_probe(force: bool = False) -> str:
    """The bench-only FP64 FMA micro-benchmark library (one source file)."""
    out, src = probe_path(), os.path.join(CSRC, PROBE_SOURCE)
    if not force and os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    cmd = [NVCC, "-shared", src, "-o", out, "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden"] + ARCH
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {PROBE_SOURCE}:\n{r.stdout}\n{r.stderr}")
    return out


def _flags(prec: str):
    f = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden,-O2", "-I", CSRC] + ARCH
    if prec == "sp":
        f += ["-DCFD2LCS_SP"]
    f += os.environ.get("CFD2LCS_B200_NVCC_FLAGS", "").split()
    return f


def _newest_input() -> float:
    files = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.abspath(__file__)]
    return max(os.path.getmtime(p) for p in files if os.path.exists(p))


def _compile(src: str, obj: str, prec: str):
    cmd = [NVCC, "-c", os.path.join(CSRC, src), "-o", obj] + _flags(prec)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return r.stderr


def build(precisions=("dp", "sp"), force: bool = False, verbose: bool = False) -> list:
    os.makedirs(BUILD, exist_ok=True)
    newest = _newest_input()
    jobs = []
    for prec in precisions:
        out = lib_path(prec)
        if not force and os.path.exists(out) and os.path.getmtime(out) >= newest:
            continue
        jobs.append(prec)
    if not jobs:
        return [lib_path(p) for p in precisions]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        futs = {}
        for prec in jobs:
            for src in SOURCES:
                obj = os.path.join(BUILD, f"{os.path.splitext(src)[0]}_{prec}.o")
                futs[ex.submit(_compile, src, obj, prec)] = (prec, src)
        for f in cf.as_completed(futs):
            err = f.result()
            if verbose and err.strip():
                print(err, file=sys.stderr)
    for prec in jobs:
        objs = [os.path.join(BUILD, f"{os.path.splitext(s)[0]}_{prec}.o") for s in SOURCES]
        cmd = [NVCC, "-shared", "-o", lib_path(prec)] + objs + ARCH + ["-Xcompiler", "-fPIC"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return [lib_path(p) for p in precisions]


if __name__ == "__main__":
    precs = tuple(a for a in sys.argv[1:] if a in ("dp", "sp")) or ("dp", "sp")
    print(build(precs, force="--force" in sys.argv, verbose=True))
    print(build_probe(force="--force" in sys.argv))
