"""ctypes binding of oracle/_cpu/libns3d_cpu.so (TEST INFRASTRUCTURE).

The library is this project's C++ / OpenMP restatement of the RK3 step
(oracle/cpu_rk3.cpp), built by ``make -C oracle cpu``: the second form of
the checker and the host-core baseline of bench.py.  Needs no GPU.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_cpu", "libns3d_cpu.so")
_dp = ctypes.POINTER(ctypes.c_double)
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def _load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(LIB_PATH)
        lib.cpu_rk3_create.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 3
        lib.cpu_rk3_create.restype = ctypes.c_void_p
        lib.cpu_rk3_destroy.argtypes = [ctypes.c_void_p]
        lib.cpu_rk3_threads.restype = ctypes.c_int
        lib.cpu_rk3_set_forcing.argtypes = [ctypes.c_void_p, _dp]
        lib.cpu_rk3_steps.argtypes = [ctypes.c_void_p, _dp, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_int]
        lib.cpu_convolution.argtypes = [ctypes.c_void_p, _dp, _dp]
        _lib = lib
    return _lib


class CpuRK3:
    """One grid of the C++ restatement; fields are lists of 3 complex128
    arrays of shape (Nx, Ny, Nz//2+1)."""

    def __init__(self, Nx, Ny, Nz, Lx=2 * np.pi, Ly=2 * np.pi, Lz=2 * np.pi):
        self.lib = _load()
        self.shape = (3, Nx, Ny, Nz // 2 + 1)
        self.h = self.lib.cpu_rk3_create(Nx, Ny, Nz, Lx, Ly, Lz)
        if not self.h:
            raise ValueError("unsupported grid extent for the CPU FFT (2^a 3^b only)")

    @property
    def threads(self) -> int:
        return int(self.lib.cpu_rk3_threads())

    def close(self):
        if self.h:
            self.lib.cpu_rk3_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _pack(self, U):
        a = np.ascontiguousarray(np.stack([np.asarray(u, dtype=np.complex128) for u in U]))
        assert a.shape == self.shape
        return a

    def set_forcing(self, F):
        a = self._pack(F)
        self.lib.cpu_rk3_set_forcing(self.h, a.view(np.float64).ctypes.data_as(_dp))

    def rk3_ssp(self, U, dt, Re, nsteps=1):
        a = self._pack(U)
        self.lib.cpu_rk3_steps(self.h, a.view(np.float64).ctypes.data_as(_dp), dt, Re, nsteps)
        return list(a)

    def convolution(self, U):
        a = self._pack(U)
        out = np.zeros(self.shape, dtype=np.complex128)
        self.lib.cpu_convolution(self.h, a.view(np.float64).ctypes.data_as(_dp),
                                 out.view(np.float64).ctypes.data_as(_dp))
        return list(out)
