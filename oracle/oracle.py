"""ctypes front end of the oracle (TEST INFRASTRUCTURE ONLY).

Loads ``liboracle_dp.so`` / ``liboracle_sp.so`` built from ``cfd2lcs_oracle.c`` (the CPU
restatement of libcfd2lcs's single-rank hot path).  Only tests, ``__graft_entry__.smoke``
and ``bench.py``'s CPU-baseline / reference arm use it -- as the checker, never as the
product.  Parity of this oracle is unpinned: the reference has no tests or golden data
and cannot be built here.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def build() -> None:
    """Compile both precisions with oracle/Makefile (gcc, no FMA contraction)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


class Oracle:
    """One oracle instance == one process-global reference state (like the Fortran
    module globals).  Two Oracle objects of the same precision share that state."""

    def __init__(self, precision: str = "dp"):
        assert precision in ("dp", "sp")
        path = os.path.join(HERE, f"liboracle_{precision}.so")
        if not os.path.exists(path):
            build()
        self.lib = C.CDLL(path)
        self.dtype = np.float64 if precision == "dp" else np.float32
        R = C.c_double if precision == "dp" else C.c_float
        self.R = R
        P = C.c_void_p
        L = self.lib
        L.orc_real_size.restype = C.c_int
        L.orc_error.restype = C.c_int
        L.orc_error_msg.restype = C.c_char_p
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_get_threads.restype = C.c_int
        L.orc_reset.restype = None
        L.orc_init.argtypes = [P, P, P, P, P, P]
        L.orc_diagnostic_init.argtypes = [C.c_int, C.c_int, R, R, C.c_char_p]
        L.orc_diagnostic_init.restype = C.c_int
        L.orc_update.argtypes = [P, P, P, P, R]
        L.orc_set_option.argtypes = [C.c_char_p, C.c_int]
        L.orc_set_param.argtypes = [C.c_char_p, R]
        L.orc_get_ftle.argtypes = [C.c_int, P]
        L.orc_get_ftle.restype = C.c_int
        L.orc_get_fm.argtypes = [C.c_int, P, C.c_int]
        L.orc_get_fm.restype = C.c_int
        L.orc_get_invariants.argtypes = [C.c_int, P]
        L.orc_get_invariants.restype = C.c_int
        L.orc_set_output_dir.argtypes = [C.c_char_p]
        L.orc_diag_size.argtypes = [C.c_int, P]
        L.orc_diag_size.restype = C.c_int
        L.orc_tracer_count.argtypes = [C.c_int]
        L.orc_tracer_count.restype = C.c_int
        L.orc_get_tracers.argtypes = [C.c_int, P]
        L.orc_get_tracers.restype = C.c_int
        L.orc_get_l2margin.argtypes = [C.c_int, P]
        L.orc_get_l2margin.restype = C.c_int
        L.orc_get_particles.argtypes = [C.c_int, P]
        L.orc_get_particles.restype = C.c_int
        L.orc_counter.argtypes = [C.c_int]
        L.orc_counter.restype = C.c_longlong
        L.orc_padded_size.restype = C.c_long
        L.orc_get_grid.argtypes = [P, P, P, P, P]
        L.orc_get_lsq_weights.argtypes = [P]
        L.orc_get_lsq_weights.restype = C.c_int
        L.orc_eig3_max.argtypes = [P]
        L.orc_eig3_max.restype = C.c_double
        L.orc_bspline3.argtypes = [P, P, P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P, C.c_int, P, P, P, P]
        L.orc_bspline3.restype = C.c_int
        L.orc_bspline3_coef.argtypes = [P, P, P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P, P]
        L.orc_bspline3_coef.restype = C.c_int
        L.orc_interp_points.argtypes = [C.c_int, P, C.c_int, P, P, P]
        L.orc_interp_points.restype = C.c_int
        assert L.orc_real_size() == np.dtype(self.dtype).itemsize
        self.n = None

    # --- helpers -------------------------------------------------------------------
    def _r(self, a):
        return np.ascontiguousarray(a, dtype=self.dtype)

    @staticmethod
    def _p(a):
        return a.ctypes.data_as(C.c_void_p)

    # --- reference-shaped API --------------------------------------------------------
    def reset(self):
        self.lib.orc_reset()
        self.n = None

    def set_threads(self, n: int):
        self.lib.orc_set_threads(int(n))

    def threads(self) -> int:
        return self.lib.orc_get_threads()

    def init(self, n, x, y, z, flag, offset=(0, 0, 0)):
        n = np.ascontiguousarray(n, dtype=np.int32)
        off = np.ascontiguousarray(offset, dtype=np.int32)
        x, y, z = self._r(x.ravel(order="F")), self._r(y.ravel(order="F")), self._r(z.ravel(order="F"))
        f = np.ascontiguousarray(flag.ravel(order="F"), dtype=np.int32)
        self.lib.orc_init(self._p(n), self._p(off), self._p(x), self._p(y), self._p(z), self._p(f))
        self.n = tuple(int(v) for v in n)

    def diagnostic_init(self, lcs_type, resolution, T, h, label="lcs"):
        return self.lib.orc_diagnostic_init(int(lcs_type), int(resolution), self.R(T), self.R(h), label.encode())

    def update(self, u, v, w, time):
        n = np.ascontiguousarray(self.n, dtype=np.int32)
        u, v, w = self._r(u.ravel(order="F")), self._r(v.ravel(order="F")), self._r(w.ravel(order="F"))
        self.lib.orc_update(self._p(n), self._p(u), self._p(v), self._p(w), self.R(time))

    def set_option(self, name, val):
        self.lib.orc_set_option(name.encode(), int(val))

    def set_param(self, name, val):
        self.lib.orc_set_param(name.encode(), self.R(val))

    def error(self) -> int:
        return self.lib.orc_error()

    def error_msg(self) -> str:
        return self.lib.orc_error_msg().decode()

    def diag_size(self, handle):
        """Grid points per direction of a diagnostic's lcs grid (resolution /= 0 changes it)."""
        n = np.zeros(3, dtype=np.int32)
        assert self.lib.orc_diag_size(handle, n.ctypes.data_as(C.c_void_p)) == 0
        return tuple(int(v) for v in n)

    def ftle(self, handle):
        n = self.diag_size(handle)
        out = np.zeros(int(np.prod(n)), dtype=self.dtype)
        assert self.lib.orc_get_ftle(handle, self._p(out)) == 0
        return out.reshape(n, order="F")

    def flowmap(self, handle, composed: bool = True):
        """composed=True: the T flow map of the last FTLE frame; False: the working map."""
        n = self.diag_size(handle)
        out = np.zeros(3 * int(np.prod(n)), dtype=self.dtype)
        assert self.lib.orc_get_fm(handle, self._p(out), int(composed)) == 0
        return out.reshape((3,) + tuple(n[::-1])).transpose(0, 3, 2, 1)

    def invariants(self, handle):
        """Q, D, C, H, L2 of the last frame (compute_invariants), shape (5, ni, nj, nk)."""
        n = self.diag_size(handle)
        out = np.zeros(5 * int(np.prod(n)), dtype=self.dtype)
        assert self.lib.orc_get_invariants(handle, self._p(out)) == 0
        return out.reshape((5,) + tuple(n[::-1])).transpose(0, 3, 2, 1)

    def tracers(self, handle):
        """Positions of an LP_TRACER set, shape (3, count)."""
        n = int(self.lib.orc_tracer_count(int(handle)))
        assert n >= 0
        out = np.zeros(3 * n, dtype=self.dtype)
        assert self.lib.orc_get_tracers(int(handle), self._p(out)) == 0
        return out.reshape(3, n)

    def set_output_dir(self, path: str):
        """Directory of the write_lcs files (WRITE_LCS); the reference's ./cfd2lcs_output."""
        self.lib.orc_set_output_dir(str(path).encode())

    def l2margin(self, handle):
        """Middle eigenvalue of the lambda-2 tensor over its largest magnitude, last frame."""
        n = self.diag_size(handle)
        out = np.zeros(int(np.prod(n)), dtype=self.dtype)
        assert self.lib.orc_get_l2margin(handle, self._p(out)) == 0
        return out.reshape(tuple(n[::-1])).transpose(2, 1, 0)

    def particles(self, handle):
        out = np.zeros(3 * int(np.prod(self.n)), dtype=self.dtype)
        assert self.lib.orc_get_particles(handle, self._p(out)) == 0
        return out.reshape(3, -1)

    def counter(self, which: str) -> int:
        idx = {"integrations_fwd": 0, "integrations_bkwd": 1, "nsub_fwd": 2, "nsub_bkwd": 3, "ftle_frames": 4}[which]
        return int(self.lib.orc_counter(idx))

    def grid_state(self):
        nt = int(self.lib.orc_padded_size())
        xyz = np.zeros(3 * nt, dtype=self.dtype)
        flag = np.zeros(nt, dtype=np.int32)
        nrm = np.zeros(3 * nt, dtype=self.dtype)
        inv = np.zeros(3 * nt, dtype=self.dtype)
        per = np.zeros(3, dtype=np.int32)
        self.lib.orc_get_grid(self._p(xyz), self._p(flag), self._p(nrm), self._p(inv), self._p(per))
        shp = tuple(v + 2 for v in self.n[::-1])
        return dict(
            xyz=xyz.reshape((3,) + shp).transpose(0, 3, 2, 1),
            flag=flag.reshape(shp).transpose(2, 1, 0),
            bcnorm=nrm.reshape((3,) + shp).transpose(0, 3, 2, 1),
            inv_delta=inv.reshape((3,) + shp).transpose(0, 3, 2, 1),
            periodic=per.astype(bool),
        )

    def lsq_weights(self):
        """(rectilinear, weights): compute_lsgw's face-neighbour weights, shape
        (6 neighbours, 3 components, ni+2, nj+2, nk+2); zeros on a rectilinear grid."""
        nt = int(self.lib.orc_padded_size())
        w = np.zeros(18 * nt, dtype=self.dtype)
        rect = int(self.lib.orc_get_lsq_weights(self._p(w)))
        shp = tuple(v + 2 for v in self.n[::-1])
        return bool(rect), w.reshape((6, 3) + shp).transpose(0, 1, 4, 3, 2)

    # --- unit helpers ----------------------------------------------------------------
    def eig3_max(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(9)
        return self.lib.orc_eig3_max(self._p(a))

    def bspline3(self, xg, yg, zg, f, order, pts):
        xg, yg, zg = self._r(xg), self._r(yg), self._r(zg)
        f = self._r(np.asarray(f).ravel(order="F"))
        pts = np.asarray(pts, dtype=self.dtype)
        px, py, pz = (self._r(pts[:, a]) for a in range(3))
        out = np.zeros(len(pts), dtype=self.dtype)
        kx, ky, kz = order
        rc = self.lib.orc_bspline3(self._p(xg), self._p(yg), self._p(zg), len(xg), len(yg), len(zg), kx, ky, kz, self._p(f),
                                   len(pts), self._p(px), self._p(py), self._p(pz), self._p(out))
        assert rc == 0
        return out

    def interp_points(self, method, f3, pts, nodes):
        """interp_s2u_r1 on the initialised grid: f3 (3, n1+2, n2+2, n3+2) padded fields, pts
        (3, np) positions, nodes (3, np) padded node indices; returns (3, np)."""
        f = np.ascontiguousarray(np.asarray(f3, dtype=self.dtype).transpose(0, 3, 2, 1)).ravel()
        p = np.ascontiguousarray(np.asarray(pts, dtype=self.dtype))
        q = np.ascontiguousarray(np.asarray(nodes, dtype=np.int32))
        out = np.zeros(p.shape, dtype=self.dtype)
        rc = self.lib.orc_interp_points(int(method), self._p(f), p.shape[1], self._p(p), self._p(q), self._p(out))
        if rc:
            raise RuntimeError(self.error_msg())
        return out

    def bspline3_coef(self, xg, yg, zg, f, order):
        xg, yg, zg = self._r(xg), self._r(yg), self._r(zg)
        f = self._r(np.asarray(f).ravel(order="F"))
        out = np.zeros_like(f)
        kx, ky, kz = order
        rc = self.lib.orc_bspline3_coef(self._p(xg), self._p(yg), self._p(zg), len(xg), len(yg), len(zg), kx, ky, kz, self._p(f),
                                        self._p(out))
        assert rc == 0
        return out.reshape((len(xg), len(yg), len(zg)), order="F")
