"""ctypes binding of oracle/_ref/libns3d_ref[_compat].so (TEST INFRASTRUCTURE).

The library is the reference's own CUDA path (unmodified sources, built for
sm_100a by oracle/Makefile) plus the project-written harness
oracle/ref_harness.cu.  Only tests/, the golden-vector generator and the
reference arm of bench.py load it.  It needs a GPU.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libns3d_ref.so")

_dp = ctypes.POINTER(ctypes.c_double)


def available() -> bool:
    return os.path.exists(LIB_PATH)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


COMPAT_LIB_PATH = os.path.join(_HERE, "_ref", "libns3d_ref_compat.so")


class RefSolver:
    """One instance of the reference's file-static state (it is not re-entrant).

    ``lib_path`` selects the build of the harness: the default links the
    reference's own objects; COMPAT_LIB_PATH links the same harness object
    against this project's reference-signature layer (libns3d_compat.so).
    """

    _libs = {}

    def __init__(self, Nx, Ny, Nz, Lx=2 * np.pi, Ly=2 * np.pi, Lz=2 * np.pi, lib_path=None):
        path = lib_path or LIB_PATH
        if path not in RefSolver._libs:
            lib = ctypes.CDLL(path)
            for name in ("ref_set_u", "ref_set_v", "ref_set_f", "ref_get_u", "ref_get_v",
                         "ref_conv", "ref_conv_uv"):
                getattr(lib, name).argtypes = [_dp]
                getattr(lib, name).restype = ctypes.c_int
            lib.ref_create.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 3
            lib.ref_create.restype = ctypes.c_int
            lib.ref_destroy.restype = None
            lib.ref_rk3.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double]
            lib.ref_jvp.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double]
            lib.ref_euler.argtypes = [ctypes.c_double, ctypes.c_double]
            lib.ref_linrhs.argtypes = [ctypes.c_double, ctypes.c_double]
            lib.ref_iuv.argtypes = [ctypes.c_double, ctypes.c_double]
            lib.ref_rhs.argtypes = [ctypes.c_double, _dp]
            lib.ref_c2r.argtypes = [_dp, _dp]
            lib.ref_r2c.argtypes = [_dp, _dp]
            lib.ref_diag.argtypes = [_dp, _dp]
            lib.ref_time_rk3.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double]
            lib.ref_time_rk3.restype = ctypes.c_double
            lib.ref_diag_record.argtypes = [ctypes.c_double, ctypes.c_double, _dp, ctypes.c_int]
            lib.ref_filters.argtypes = [ctypes.c_double, ctypes.c_double, _dp, _dp]
            lib.ref_curl.argtypes = [_dp, _dp]
            lib.ref_shapiro_error.argtypes = [ctypes.c_double, ctypes.c_double, _dp]
            lib.ref_u_ptr.argtypes = [ctypes.c_int]
            lib.ref_u_ptr.restype = ctypes.c_void_p
            RefSolver._libs[path] = lib
        self.lib = RefSolver._libs[path]
        self.Nx, self.Ny, self.Nz = Nx, Ny, Nz
        self.Mz = Nz // 2 + 1
        rc = self.lib.ref_create(Nx, Ny, Nz, Lx, Ly, Lz)
        if rc != 0:
            raise RuntimeError(f"ref_create failed ({rc})")

    def close(self):
        self.lib.ref_destroy()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # field helpers --------------------------------------------------------
    def _pack(self, U):
        a = np.ascontiguousarray(np.stack([np.asarray(u, dtype=np.complex128) for u in U]))
        assert a.shape == (3, self.Nx, self.Ny, self.Mz)
        return a.view(np.float64)

    def _empty(self):
        return np.zeros((3, self.Nx, self.Ny, self.Mz), dtype=np.complex128)

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed ({rc})")

    def set_u(self, U):
        a = self._pack(U)
        self._check(self.lib.ref_set_u(_ptr(a)), "set_u")

    def set_v(self, V):
        a = self._pack(V)
        self._check(self.lib.ref_set_v(_ptr(a)), "set_v")

    def set_f(self, F):
        a = self._pack(F)
        self._check(self.lib.ref_set_f(_ptr(a)), "set_f")

    def get_u(self):
        out = self._empty()
        self._check(self.lib.ref_get_u(_ptr(out.view(np.float64))), "get_u")
        return list(out)

    def get_v(self):
        out = self._empty()
        self._check(self.lib.ref_get_v(_ptr(out.view(np.float64))), "get_v")
        return list(out)

    # reference entry points ----------------------------------------------
    def rk3(self, nsteps, dt, Re):
        self._check(self.lib.ref_rk3(nsteps, dt, Re), "rk3")

    def euler(self, dt, Re):
        self._check(self.lib.ref_euler(dt, Re), "euler")

    def jvp(self, nsteps, dt, Re):
        self._check(self.lib.ref_jvp(nsteps, dt, Re), "jvp")

    def linrhs(self, dt, Re):
        self._check(self.lib.ref_linrhs(dt, Re), "linrhs")

    def iuv(self, dt, Re):
        self._check(self.lib.ref_iuv(dt, Re), "iuv")

    def rhs(self, Re):
        out = self._empty()
        self._check(self.lib.ref_rhs(Re, _ptr(out.view(np.float64))), "rhs")
        return list(out)

    def conv(self):
        out = self._empty()
        self._check(self.lib.ref_conv(_ptr(out.view(np.float64))), "conv")
        return list(out)

    def conv_uv(self):
        out = self._empty()
        self._check(self.lib.ref_conv_uv(_ptr(out.view(np.float64))), "conv_uv")
        return list(out)

    def c2r(self, X):
        X = np.ascontiguousarray(X, dtype=np.complex128)
        out = np.zeros((self.Nx, self.Ny, self.Nz))
        self._check(self.lib.ref_c2r(_ptr(X.view(np.float64)), _ptr(out)), "c2r")
        return out

    def r2c(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.zeros((self.Nx, self.Ny, self.Mz), dtype=np.complex128)
        self._check(self.lib.ref_r2c(_ptr(x), _ptr(out.view(np.float64))), "r2c")
        return out

    def diag(self):
        e = np.zeros(1)
        d = np.zeros(1)
        self._check(self.lib.ref_diag(_ptr(e), _ptr(d)), "diag")
        return float(e[0]), float(d[0])

    def record(self, total_time, Re, preserve=True):
        """The main loop's 50-column record.  preserve=False transforms the
        state arrays in place as main does (cuFFT may overwrite them; get_u
        shows what is left); preserve=True transforms a copy."""
        rec = np.zeros(50)
        self._check(self.lib.ref_diag_record(total_time, Re, _ptr(rec), int(bool(preserve))),
                    "record")
        return rec

    def filters(self, eps, radius):
        """Physical velocities of the Helmholtz (eps) and cut-off (radius)
        filtered state."""
        ph = np.zeros((3, self.Nx, self.Ny, self.Nz))
        pc = np.zeros((3, self.Nx, self.Ny, self.Nz))
        self._check(self.lib.ref_filters(eps, radius, _ptr(ph), _ptr(pc)), "filters")
        return ph, pc

    def curl(self, u):
        a = np.ascontiguousarray(np.stack([np.asarray(x, dtype=np.float64) for x in u]))
        r = np.zeros_like(a)
        self._check(self.lib.ref_curl(_ptr(a), _ptr(r)), "curl")
        return r

    def shapiro_error(self, t, Re):
        e = np.zeros(1)
        self._check(self.lib.ref_shapiro_error(t, Re, _ptr(e)), "shapiro_error")
        return float(e[0])

    def time_rk3(self, nsteps, dt, Re):
        ms = self.lib.ref_time_rk3(nsteps, dt, Re)
        if ms < 0:
            raise RuntimeError("time_rk3 failed")
        return ms
