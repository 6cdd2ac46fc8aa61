"""libcfd2lcs_b200 -- B200-native (sm_100a) FTLE hot path of libcfd2lcs behind its C ABI.

The product is the shared library ``libcfd2lcs_b200_{dp,sp}.so`` (C / Fortran entry points
of the reference, see include/cfd2lcs_inc_dp.h).  This module is the Python mirror of that
interface, for tests, benchmarks and Python drivers: the same call names, argument meaning
and error behaviour as the reference's cfd2lcs_* entry points (src/cfd2lcs_c.c:67-142).

There is no CPU fallback: every call goes through the CUDA library, which latches an error
(like the reference's CFD2LCS_ERROR) when no GPU is available.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np


HERE = os.path.dirname(os.path.abspath(__file__))

# constants of cfd2lcs_inc_double.h:27-65
LCS_INTERNAL, LCS_INFLOW, LCS_OUTFLOW, LCS_WALL, LCS_SLIP, LCS_2D, LCS_MASK = range(7)
FTLE_FWD, FTLE_BKWD, LP_TRACER = 0, 1, 2
EULER, TRAPEZOIDAL, RK2, RK3, RK4 = 0, 1, 2, 3, 4
NEAREST_NBR, LINEAR, QUADRATIC, CUBIC, TSE, TSE_LIMIT = 0, 1, 2, 3, 5, 6
LCS_FALSE, LCS_TRUE = 0, 1
LCS_NAMELEN = 128

EXPORTED_SYMBOLS = [
    # reference C interface (src/cfd2lcs_c.c)
    "cfd2lcs_init_c", "cfd2lcs_diagnostic_init_c", "cfd2lcs_update_c", "cfd2lcs_diagnostic_destroy_c",
    "cfd2lcs_set_option_c", "cfd2lcs_set_param_c",
    # reference Fortran interface (src/cfd2lcs.f90), gfortran mangling
    "cfd2lcs_init_", "cfd2lcs_diagnostic_init_", "cfd2lcs_update_", "cfd2lcs_diagnostic_destroy_",
    "cfd2lcs_set_option_", "cfd2lcs_set_param_", "cfd2lcs_finalize_",
    # extensions (include/cfd2lcs_b200.h)
    "cfd2lcs_finalize_c", "cfd2lcs_get_error_c", "cfd2lcs_reset_c", "cfd2lcs_get_ftle_c", "cfd2lcs_get_flowmap_c",
    "cfd2lcs_update_device_c", "cfd2lcs_ftle_device_ptr_c", "cfd2lcs_get_counters_c", "cfd2lcs_get_phase_times_c",
    "cfd2lcs_get_kernel_times_c", "cfd2lcs_get_staged_launches_c", "cfd2lcs_get_march_launches_c", "cfd2lcs_get_tuning_c", "cfd2lcs_reconstruct_noalloc_c", "cfd2lcs_get_invariants_c",
    "cfd2lcs_tracer_count_c", "cfd2lcs_get_tracers_c", "cfd2lcs_diagnostic_size_c",
    # batched form (include/cfd2lcs_b200.h)
    "cfd2lcs_batch_add_c", "cfd2lcs_batch_diagnostic_init_c", "cfd2lcs_batch_update_device_c", "cfd2lcs_batch_get_ftle_c",
    "cfd2lcs_batch_get_flowmap_c", "cfd2lcs_batch_get_counters_c", "cfd2lcs_batch_size_c", "cfd2lcs_batch_error_c",
    "cfd2lcs_batch_reset_c",
    # adjoint (include/cfd2lcs_b200.h)
    "cfd2lcs_adjoint_ftle_c", "cfd2lcs_tangent_ftle_c", "cfd2lcs_adjoint_ftle_interp_c", "cfd2lcs_tangent_ftle_interp_c",
    # measurement hook (include/cfd2lcs_b200.h)
]


def library_path(precision: str = "dp") -> str:
    """In-tree library, or the one in $CFD2LCS_B200_LIBDIR when that is set."""
    d = os.environ.get("CFD2LCS_B200_LIBDIR") or HERE
    return os.path.join(d, f"libcfd2lcs_b200_{precision}.so")


def build(precisions=("dp", "sp"), force=False):
    from .build import build as _b
    return _b(precisions, force=force)


_LIBS = {}


def load(precision: str = "dp") -> C.CDLL:
    """Loads the in-tree CUDA library; raises if it has not been built (no fallback)."""
    if precision in _LIBS:
        return _LIBS[precision]
    path = library_path(precision)
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m libcfd2lcs_b200.build` (no CPU fallback exists)")
    lib = C.CDLL(path)
    R = C.c_double if precision == "dp" else C.c_float
    P = C.c_void_p
    lib.cfd2lcs_init_c.argtypes = [C.c_ssize_t, P, P, P, P, P, P]
    lib.cfd2lcs_init_c.restype = None
    lib.cfd2lcs_diagnostic_init_c.argtypes = [C.c_int, C.c_int, R, R, C.c_char_p]
    lib.cfd2lcs_diagnostic_init_c.restype = C.c_int
    lib.cfd2lcs_update_c.argtypes = [P, P, P, P, R]
    lib.cfd2lcs_update_c.restype = None
    lib.cfd2lcs_update_device_c.argtypes = [P, P, P, P, R]
    lib.cfd2lcs_update_device_c.restype = None
    lib.cfd2lcs_diagnostic_destroy_c.argtypes = [C.c_int]
    lib.cfd2lcs_set_option_c.argtypes = [C.c_char_p, C.c_int]
    lib.cfd2lcs_set_param_c.argtypes = [C.c_char_p, R]
    lib.cfd2lcs_finalize_c.restype = None
    lib.cfd2lcs_reset_c.restype = None
    lib.cfd2lcs_get_error_c.argtypes = [C.c_char_p, C.c_size_t]
    lib.cfd2lcs_get_error_c.restype = C.c_int
    lib.cfd2lcs_get_ftle_c.argtypes = [C.c_int, P]
    lib.cfd2lcs_get_ftle_c.restype = C.c_int
    lib.cfd2lcs_get_flowmap_c.argtypes = [C.c_int, P]
    lib.cfd2lcs_get_flowmap_c.restype = C.c_int
    lib.cfd2lcs_get_invariants_c.argtypes = [C.c_int, P]
    lib.cfd2lcs_get_invariants_c.restype = C.c_int
    lib.cfd2lcs_diagnostic_size_c.argtypes = [C.c_int, P]
    lib.cfd2lcs_diagnostic_size_c.restype = C.c_int
    lib.cfd2lcs_tracer_count_c.argtypes = [C.c_int]
    lib.cfd2lcs_tracer_count_c.restype = C.c_int
    lib.cfd2lcs_get_tracers_c.argtypes = [C.c_int, P]
    lib.cfd2lcs_get_tracers_c.restype = C.c_int
    lib.cfd2lcs_ftle_device_ptr_c.argtypes = [C.c_int]
    lib.cfd2lcs_ftle_device_ptr_c.restype = C.c_void_p
    lib.cfd2lcs_get_counters_c.argtypes = [P]
    lib.cfd2lcs_get_phase_times_c.argtypes = [P]
    lib.cfd2lcs_get_kernel_times_c.argtypes = [P, P]
    lib.cfd2lcs_get_staged_launches_c.argtypes = [P]
    lib.cfd2lcs_get_march_launches_c.argtypes = [P]
    lib.cfd2lcs_get_tuning_c.argtypes = [P, P]
    lib.cfd2lcs_reconstruct_noalloc_c.argtypes = [C.c_int, P, P]
    lib.cfd2lcs_reconstruct_noalloc_c.restype = C.c_int
    lib.cfd2lcs_b200_grid_tables.argtypes = [P, P, P, P, P, P, P, P, P, P, C.c_char_p, C.c_size_t]
    lib.cfd2lcs_b200_grid_tables.restype = C.c_int
    lib.cfd2lcs_b200_grid_lsq_weights.argtypes = [P, P, P, P, P, P, P, C.c_char_p, C.c_size_t]
    lib.cfd2lcs_b200_grid_lsq_weights.restype = C.c_int
    lib.cfd2lcs_batch_add_c.argtypes = [P, P, P, P, P, C.c_int, C.c_int, R, C.c_int]
    lib.cfd2lcs_batch_add_c.restype = C.c_int
    lib.cfd2lcs_batch_diagnostic_init_c.argtypes = [C.c_int, C.c_int, R, R]
    lib.cfd2lcs_batch_diagnostic_init_c.restype = C.c_int
    lib.cfd2lcs_batch_update_device_c.argtypes = [C.c_int, P, P, P, P, P]
    lib.cfd2lcs_batch_update_device_c.restype = C.c_int
    for f in (lib.cfd2lcs_batch_get_ftle_c, lib.cfd2lcs_batch_get_flowmap_c):
        f.argtypes = [C.c_int, C.c_int, P]
        f.restype = C.c_int
    lib.cfd2lcs_batch_get_counters_c.argtypes = [C.c_int, P]
    lib.cfd2lcs_batch_get_counters_c.restype = C.c_int
    lib.cfd2lcs_batch_size_c.restype = C.c_int
    lib.cfd2lcs_batch_error_c.argtypes = [C.c_char_p, C.c_size_t]
    lib.cfd2lcs_batch_error_c.restype = C.c_int
    lib.cfd2lcs_batch_reset_c.restype = None
    lib.cfd2lcs_adjoint_ftle_c.argtypes = [P, P, P, P, C.c_int, R, C.c_int, P, P, P, P, P, C.c_int, P, P, P, P, C.c_char_p, C.c_size_t]
    lib.cfd2lcs_adjoint_ftle_c.restype = C.c_int
    lib.cfd2lcs_tangent_ftle_c.argtypes = [P, P, P, P, C.c_int, R, C.c_int, P, P, P, P, P, P, P, P, P, P, C.c_char_p, C.c_size_t]
    lib.cfd2lcs_tangent_ftle_c.restype = C.c_int
    lib.cfd2lcs_adjoint_ftle_interp_c.argtypes = [P, P, P, P, P, C.c_int, C.c_int, R, C.c_int, P, P, P, P, P, C.c_int, P, P, P, P,
                                                  C.c_char_p, C.c_size_t]
    lib.cfd2lcs_adjoint_ftle_interp_c.restype = C.c_int
    lib.cfd2lcs_tangent_ftle_interp_c.argtypes = [P, P, P, P, P, C.c_int, C.c_int, R, C.c_int, P, P, P, P, P, P, P, P, P, P,
                                                  C.c_char_p, C.c_size_t]
    lib.cfd2lcs_tangent_ftle_interp_c.restype = C.c_int
    _LIBS[precision] = lib
    return lib


class Cfd2lcs:
    """The reference's entry points on one library instance (process-global state, like the
    Fortran module globals).  Arrays are numpy arrays of shape (ni, nj, nk); they are
    passed in Fortran (i-fastest) order."""

    def __init__(self, precision: str = "dp"):
        self.precision = precision
        self.lib = load(precision)
        self.dtype = np.float64 if precision == "dp" else np.float32
        self.R = C.c_double if precision == "dp" else C.c_float
        self.n = None

    @staticmethod
    def _p(a):
        return a.ctypes.data_as(C.c_void_p)

    def _r(self, a):
        return np.asfortranarray(a, dtype=self.dtype).ravel(order="F")

    # reference API ---------------------------------------------------------------------
    def init(self, n, x, y, z, flag, offset=(0, 0, 0), comm: int = 0):
        n = np.ascontiguousarray(n, dtype=np.int32)
        off = np.ascontiguousarray(offset, dtype=np.int32)
        x, y, z = self._r(x), self._r(y), self._r(z)
        f = np.asfortranarray(flag, dtype=np.int32).ravel(order="F")
        self.lib.cfd2lcs_init_c(comm, self._p(n), self._p(off), self._p(x), self._p(y), self._p(z), self._p(f))
        self.n = tuple(int(v) for v in n)

    def diagnostic_init(self, lcs_type, resolution, T, h, label="lcs") -> int:
        return self.lib.cfd2lcs_diagnostic_init_c(int(lcs_type), int(resolution), self.R(T), self.R(h), label.encode())

    def update(self, u, v, w, time):
        n = np.ascontiguousarray(self.n if self.n else (0, 0, 0), dtype=np.int32)
        u, v, w = self._r(u), self._r(v), self._r(w)
        self.lib.cfd2lcs_update_c(self._p(n), self._p(u), self._p(v), self._p(w), self.R(time))

    def update_device(self, d_u: int, d_v: int, d_w: int, time):
        """u, v, w already in device memory (raw device pointers, e.g. tensor.data_ptr())."""
        n = np.ascontiguousarray(self.n, dtype=np.int32)
        self.lib.cfd2lcs_update_device_c(self._p(n), C.c_void_p(d_u), C.c_void_p(d_v), C.c_void_p(d_w), self.R(time))

    def diagnostic_destroy(self, handle):
        self.lib.cfd2lcs_diagnostic_destroy_c(int(handle))

    def set_option(self, name: str, val: int):
        self.lib.cfd2lcs_set_option_c(name.encode(), int(val))

    def set_param(self, name: str, val: float):
        self.lib.cfd2lcs_set_param_c(name.encode(), self.R(val))

    def finalize(self):
        self.lib.cfd2lcs_finalize_c()

    # extensions ------------------------------------------------------------------------
    def reset(self):
        self.lib.cfd2lcs_reset_c()
        self.n = None

    def error(self):
        buf = C.create_string_buffer(512)
        e = self.lib.cfd2lcs_get_error_c(buf, 512)
        return e, buf.value.decode()

    def diag_size(self, handle):
        """Points per direction of a diagnostic's lcs grid (differs from the grid's with
        resolution /= 0)."""
        n = np.zeros(3, dtype=np.int32)
        if self.lib.cfd2lcs_diagnostic_size_c(int(handle), self._p(n)) != 0:
            raise RuntimeError("unknown diagnostic handle")
        return tuple(int(v) for v in n)

    def ftle(self, handle):
        n = self.diag_size(handle)
        out = np.zeros(int(np.prod(n)), dtype=self.dtype)
        if self.lib.cfd2lcs_get_ftle_c(int(handle), self._p(out)) != 0:
            raise RuntimeError("no FTLE field for this handle yet")
        return out.reshape(n, order="F")

    def flowmap(self, handle):
        n = self.diag_size(handle)
        out = np.zeros(3 * int(np.prod(n)), dtype=self.dtype)
        if self.lib.cfd2lcs_get_flowmap_c(int(handle), self._p(out)) != 0:
            raise RuntimeError("no flow map for this handle yet")
        N = int(np.prod(n))
        return np.stack([out[c * N:(c + 1) * N].reshape(n, order="F") for c in range(3)])

    def invariants(self, handle):
        """Q, D, C, H, L2 of the last frame (VELOCITY_INVARIANTS), shape (5, ni, nj, nk)."""
        n = self.diag_size(handle)
        out = np.zeros(5 * int(np.prod(n)), dtype=self.dtype)
        if self.lib.cfd2lcs_get_invariants_c(int(handle), self._p(out)) != 0:
            raise RuntimeError("no invariants for this handle")
        N = int(np.prod(n))
        return np.stack([out[q * N:(q + 1) * N].reshape(n, order="F") for q in range(5)])

    def tracers(self, handle):
        """Positions of an LP_TRACER set, shape (3, count)."""
        n = self.lib.cfd2lcs_tracer_count_c(int(handle))
        if n < 0:
            raise RuntimeError("not an LP_TRACER handle")
        out = np.zeros(3 * n, dtype=self.dtype)
        if self.lib.cfd2lcs_get_tracers_c(int(handle), self._p(out)) != 0:
            raise RuntimeError("get_tracers failed")
        return out.reshape(3, n)

    def ftle_device_ptr(self, handle) -> int:
        return int(self.lib.cfd2lcs_ftle_device_ptr_c(int(handle)) or 0)

    def counters(self) -> dict:
        a = np.zeros(8, dtype=np.int64)
        self.lib.cfd2lcs_get_counters_c(self._p(a))
        keys = ["integrations_fwd", "integrations_bkwd", "nsub_fwd", "nsub_bkwd", "ftle_frames", "updates", "kernel_launches",
                "slots_composed"]
        return {k: int(v) for k, v in zip(keys, a)}

    def phase_times_ms(self) -> dict:
        a = np.zeros(7, dtype=np.float64)
        self.lib.cfd2lcs_get_phase_times_c(self._p(a))
        keys = ["ingest", "bkwd_advect", "fwd_advect", "snapshot", "compose", "ftle", "update_total"]
        return {k: float(v) for k, v in zip(keys, a)}

    def reconstruct_noalloc(self, handle, d_ftle: int, d_fm: int) -> int:
        """Latest FTLE frame recomputed into caller-owned device buffers (raw device
        pointers: n values for the FTLE, 3n for the flow map) without allocating."""
        return int(self.lib.cfd2lcs_reconstruct_noalloc_c(int(handle), C.c_void_p(d_ftle), C.c_void_p(d_fm)))

    def staged_launches(self) -> dict:
        """Launches of the subcycle kernels that staged their spline taps in shared memory."""
        n = np.zeros(2, dtype=np.int64)
        self.lib.cfd2lcs_get_staged_launches_c(self._p(n))
        m = np.zeros(1, dtype=np.int64)
        self.lib.cfd2lcs_get_march_launches_c(self._p(m))
        return {"sl": int(n[0]), "fwd": int(n[1]), "sl_march": int(m[0])}

    def tuning(self) -> dict:
        """The staged-versus-gathering choice of the backward and forward subcycle kernels (-1
        sampling or not applicable, 0 gathering, 1 staged) and the shortest launch ms measured."""
        ch = np.zeros(2, dtype=np.int32)
        ms = np.zeros(4, dtype=np.float64)
        self.lib.cfd2lcs_get_tuning_c(self._p(ch), self._p(ms))
        return {"bkwd": int(ch[0]), "fwd": int(ch[1]), "bkwd_ms": [float(ms[0]), float(ms[1])], "fwd_ms": [float(ms[2]), float(ms[3])]}

    def kernel_times(self) -> dict:
        t = np.zeros(2, dtype=np.float64)
        n = np.zeros(2, dtype=np.int64)
        self.lib.cfd2lcs_get_kernel_times_c(self._p(t), self._p(n))
        return dict(sl_ms=float(t[0]), fwd_ms=float(t[1]), sl_launches=int(n[0]), fwd_launches=int(n[1]))

    def grid_tables(self, n, x, y, z, flag):
        """Host-only grid set-up (no GPU needed): padded coordinates, flags, normals and
        inverse half spans, shapes (3, ni+2, nj+2, nk+2) etc."""
        n = np.ascontiguousarray(n, dtype=np.int32)
        x, y, z = self._r(x), self._r(y), self._r(z)
        f = np.asfortranarray(flag, dtype=np.int32).ravel(order="F")
        nt = int(np.prod(np.asarray(n) + 2))
        xyz = np.zeros(3 * nt, dtype=self.dtype)
        fl = np.zeros(nt, dtype=np.int32)
        nrm = np.zeros(3 * nt, dtype=self.dtype)
        inv = np.zeros(3 * nt, dtype=self.dtype)
        per = np.zeros(3, dtype=np.int32)
        msg = C.create_string_buffer(512)
        rc = self.lib.cfd2lcs_b200_grid_tables(self._p(n), self._p(x), self._p(y), self._p(z), self._p(f), self._p(xyz), self._p(fl),
                                               self._p(nrm), self._p(inv), self._p(per), msg, 512)
        if rc != 0:
            raise ValueError(msg.value.decode())
        shp = tuple(int(v) + 2 for v in n[::-1])
        return dict(
            xyz=xyz.reshape((3,) + shp).transpose(0, 3, 2, 1),
            flag=fl.reshape(shp).transpose(2, 1, 0),
            bcnorm=nrm.reshape((3,) + shp).transpose(0, 3, 2, 1),
            inv_delta=inv.reshape((3,) + shp).transpose(0, 3, 2, 1),
            periodic=per.astype(bool),
        )

    def grid_lsq_weights(self, n, x, y, z, flag):
        """Host-only: (curvilinear, weights) with the least-squares gradient weights of a
        non-rectilinear grid, shape (6 face neighbours, 3 derivatives, ni+2, nj+2, nk+2)."""
        n = np.ascontiguousarray(n, dtype=np.int32)
        x, y, z = self._r(x), self._r(y), self._r(z)
        f = np.asfortranarray(flag, dtype=np.int32).ravel(order="F")
        nt = int(np.prod(np.asarray(n) + 2))
        w = np.zeros(18 * nt, dtype=self.dtype)
        curv = C.c_int(0)
        msg = C.create_string_buffer(512)
        rc = self.lib.cfd2lcs_b200_grid_lsq_weights(self._p(n), self._p(x), self._p(y), self._p(z), self._p(f), self._p(w),
                                                    C.byref(curv), msg, 512)
        if rc != 0:
            raise ValueError(msg.value.decode())
        shp = tuple(int(v) + 2 for v in n[::-1])
        return bool(curv.value), w.reshape((6, 3) + shp).transpose(0, 1, 4, 3, 2)


class Batch:
    """The batched form (cfd2lcs_batch_*): independent instances, each with its own grid,
    options and diagnostics, advanced together by one call."""

    COUNTER_KEYS = ["integrations_fwd", "integrations_bkwd", "nsub_fwd", "nsub_bkwd", "ftle_frames", "updates", "kernel_launches",
                    "slots_composed"]

    def __init__(self, precision: str = "dp"):
        self.precision = precision
        self.lib = load(precision)
        self.dtype = np.float64 if precision == "dp" else np.float32
        self.R = C.c_double if precision == "dp" else C.c_float
        self.shapes = []

    def reset(self):
        self.lib.cfd2lcs_batch_reset_c()
        self.shapes = []

    def add(self, n, x, y, z, flag, integrator=2, interpolator=1, cfl=0.5, mixed=False) -> int:
        r = lambda a: np.asfortranarray(a, dtype=self.dtype).ravel(order="F")
        nn = np.ascontiguousarray(n, dtype=np.int32)
        xs, ys, zs = r(x), r(y), r(z)
        f = np.asfortranarray(flag, dtype=np.int32).ravel(order="F")
        p = lambda a: a.ctypes.data_as(C.c_void_p)
        i = self.lib.cfd2lcs_batch_add_c(p(nn), p(xs), p(ys), p(zs), p(f), int(integrator), int(interpolator), self.R(cfl),
                                         1 if mixed else 0)
        if i >= 0:
            self.shapes.append(tuple(int(v) for v in n))
        return i

    def diagnostic_init(self, inst: int, lcs_type: int, T: float, h: float) -> int:
        return self.lib.cfd2lcs_batch_diagnostic_init_c(int(inst), int(lcs_type), self.R(T), self.R(h))

    def update_device(self, ids, d_u, d_v, d_w, times) -> int:
        """ids: instance ids; d_u/d_v/d_w: device pointers (ints); times: per instance."""
        k = len(ids)
        I = np.ascontiguousarray(ids, dtype=np.int32)
        U = (C.c_void_p * k)(*d_u)
        V = (C.c_void_p * k)(*d_v)
        W = (C.c_void_p * k)(*d_w)
        Tm = np.ascontiguousarray(times, dtype=self.dtype)
        return self.lib.cfd2lcs_batch_update_device_c(k, I.ctypes.data_as(C.c_void_p), C.cast(U, C.c_void_p), C.cast(V, C.c_void_p),
                                                      C.cast(W, C.c_void_p), Tm.ctypes.data_as(C.c_void_p))

    def ftle(self, inst: int, handle: int):
        out = np.zeros(int(np.prod(self.shapes[inst])), dtype=self.dtype)
        rc = self.lib.cfd2lcs_batch_get_ftle_c(int(inst), int(handle), out.ctypes.data_as(C.c_void_p))
        if rc:
            raise RuntimeError("no FTLE field for this instance / handle")
        return out.reshape(self.shapes[inst], order="F")

    def flowmap(self, inst: int, handle: int):
        out = np.zeros(3 * int(np.prod(self.shapes[inst])), dtype=self.dtype)
        rc = self.lib.cfd2lcs_batch_get_flowmap_c(int(inst), int(handle), out.ctypes.data_as(C.c_void_p))
        if rc:
            raise RuntimeError("no flow map for this instance / handle")
        n = self.shapes[inst]
        N = int(np.prod(n))
        return np.stack([out[c * N:(c + 1) * N].reshape(n, order="F") for c in range(3)])

    def counters(self, inst: int) -> dict:
        c = np.zeros(8, dtype=np.int64)
        self.lib.cfd2lcs_batch_get_counters_c(int(inst), c.ctypes.data_as(C.c_void_p))
        return dict(zip(self.COUNTER_KEYS, (int(v) for v in c)))

    def error(self):
        buf = C.create_string_buffer(512)
        e = self.lib.cfd2lcs_batch_error_c(buf, 512)
        return int(e), buf.value.decode(errors="replace")


def adjoint_ftle(grid, u, v, w, times, weight, integrator=2, cfl=0.5, checkpoint_every=20, precision="dp", gradient=True,
                 interpolator=1):
    """J = sum(weight * FTLE) of the backward flow map over all levels and, with gradient,
    dJ/du of every level (cfd2lcs_adjoint_ftle_interp_c; interpolator 1 LINEAR or 3 CUBIC).  u, v, w: lists of CUDA tensors, one per
    level (n[0]*n[1]*n[2] values, i fastest, the library's precision); weight: CUDA tensor.
    Returns (J, gu, gv, gw) with gu, gv, gw lists of CUDA tensors (None without gradient)."""
    import torch
    lib = load(precision)
    dt = np.float64 if precision == "dp" else np.float32
    R = C.c_double if precision == "dp" else C.c_float
    L = len(u)
    n = np.ascontiguousarray(grid.n, dtype=np.int32)
    xs, ys, zs = (np.asfortranarray(a, dtype=dt).ravel(order="F") for a in (grid.x, grid.y, grid.z))
    ptrs = lambda ts: (C.c_void_p * L)(*[t.data_ptr() for t in ts])
    tm = np.ascontiguousarray(times, dtype=dt)
    J = C.c_double(0.0)
    g = None
    if gradient:
        g = [[torch.empty_like(t) for t in comp] for comp in (u, v, w)]
    msg = C.create_string_buffer(512)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    fl = np.asfortranarray(grid.flag, dtype=np.int32).ravel(order="F")
    rc = lib.cfd2lcs_adjoint_ftle_interp_c(p(n), p(xs), p(ys), p(zs), p(fl), int(integrator), int(interpolator), R(cfl), L,
                                           C.cast(ptrs(u), C.c_void_p), C.cast(ptrs(v), C.c_void_p), C.cast(ptrs(w), C.c_void_p), p(tm),
                                           C.c_void_p(weight.data_ptr()), int(checkpoint_every), C.byref(J),
                                    C.cast(ptrs(g[0]), C.c_void_p) if g else None, C.cast(ptrs(g[1]), C.c_void_p) if g else None,
                                    C.cast(ptrs(g[2]), C.c_void_p) if g else None, msg, 512)
    if rc:
        raise RuntimeError(msg.value.decode(errors="replace"))
    if g:
        return J.value, g[0], g[1], g[2]
    return J.value, None, None, None


def tangent_ftle(grid, u, v, w, times, weight, du, dv, dw, integrator=2, cfl=0.5, precision="dp", interpolator=1):
    """J and dJ = <dJ/du, d> of the adjoint's objective for one direction d = (du, dv, dw) (lists of
    CUDA tensors, one per level, like u, v, w), by the tangent-linear sweep
    (cfd2lcs_tangent_ftle_c).  Returns (J, dJ)."""
    lib = load(precision)
    dt = np.float64 if precision == "dp" else np.float32
    R = C.c_double if precision == "dp" else C.c_float
    L = len(u)
    n = np.ascontiguousarray(grid.n, dtype=np.int32)
    xs, ys, zs = (np.asfortranarray(a, dtype=dt).ravel(order="F") for a in (grid.x, grid.y, grid.z))
    ptrs = lambda ts: C.cast((C.c_void_p * L)(*[t.data_ptr() for t in ts]), C.c_void_p)
    tm = np.ascontiguousarray(times, dtype=dt)
    J, dJ = C.c_double(0.0), C.c_double(0.0)
    msg = C.create_string_buffer(512)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    fl = np.asfortranarray(grid.flag, dtype=np.int32).ravel(order="F")
    rc = lib.cfd2lcs_tangent_ftle_interp_c(p(n), p(xs), p(ys), p(zs), p(fl), int(integrator), int(interpolator), R(cfl), L, ptrs(u),
                                           ptrs(v), ptrs(w), p(tm), C.c_void_p(weight.data_ptr()), ptrs(du), ptrs(dv), ptrs(dw),
                                           C.byref(J), C.byref(dJ), msg, 512)
    if rc:
        raise RuntimeError(msg.value.decode(errors="replace"))
    return J.value, dJ.value
