"""Python host mirror of the reference's time-stepping interface.

Method names follow Source/RK_time_step.h, Source/advection_2_3.h and the
Krylov adapters of Source/NS3D_periodic.cu; each call goes through the C ABI
(include/ns3d.h) into the sm_100a kernels.  Fields are CUDA complex128
tensors of shape (Nx, Ny, Nz//2+1) in the reference layout; torch only
provides device memory and streams.
"""
from __future__ import annotations

import ctypes
import math
from typing import Sequence

from ._lib import FieldRequest, Ns3dError, Request, Result, lib

_PI2 = 2.0 * math.pi


_PRECISIONS = {"fp64": 0, "fp32": 1}


def _ptr(t) -> int:
    return int(t.data_ptr())


class Solver:
    """One ns3d_solver handle (scratch, tables, stream) on one CUDA device."""

    def __init__(self, Nx: int, Ny: int, Nz: int, Lx: float = _PI2, Ly: float = _PI2,
                 Lz: float = _PI2, device=None):
        import torch

        self._torch = torch
        dev = torch.device(device if device is not None else "cuda")
        if dev.type != "cuda":
            raise ValueError("the solver runs on CUDA devices only")
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.Nx, self.Ny, self.Nz = int(Nx), int(Ny), int(Nz)
        self.Mz = self.Nz // 2 + 1
        self.Lx, self.Ly, self.Lz = float(Lx), float(Ly), float(Lz)
        self._L = lib()
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            torch.cuda.init()
            rc = self._L.ns3d_create(self.Nx, self.Ny, self.Nz, self.Lx, self.Ly, self.Lz,
                                     ctypes.byref(h))
        if rc != 0:
            raise Ns3dError(rc, "ns3d_create")
        self._h = h
        self._forcing = None  # keeps dense forcing tensors alive

    # -- plumbing ---------------------------------------------------------
    @property
    def shape(self):
        return (self.Nx, self.Ny, self.Mz)

    def _check(self, rc: int, where: str):
        if rc != 0:
            detail = self._L.ns3d_last_error(self._h)
            raise Ns3dError(rc, where, detail.decode() if detail else "")

    def _fields(self, F: Sequence, name: str):
        torch = self._torch
        if len(F) != 3:
            raise ValueError(f"{name}: need 3 components")
        for f in F:
            if (not isinstance(f, torch.Tensor) or f.dtype != torch.complex128
                    or f.device != self.device or tuple(f.shape) != self.shape
                    or not f.is_contiguous()):
                raise ValueError(f"{name}: expected contiguous complex128 {self.shape} tensors "
                                 f"on {self.device}")
        return [_ptr(f) for f in F]

    def zeros(self):
        t = self._torch
        return [t.zeros(self.shape, dtype=t.complex128, device=self.device) for _ in range(3)]

    def to_device(self, F):
        t = self._torch
        return [t.as_tensor(f).to(device=self.device, dtype=t.complex128).contiguous() for f in F]

    def synchronize(self):
        self._check(self._L.ns3d_synchronize(self._h), "ns3d_synchronize")

    def set_stream(self, stream):
        """Use a torch.cuda.Stream (or raw handle int) for later launches."""
        raw = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        self._check(self._L.ns3d_set_stream(self._h, ctypes.c_void_p(raw)), "ns3d_set_stream")

    @property
    def device_bytes(self) -> int:
        return int(self._L.ns3d_device_bytes(self._h))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.ns3d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- forcing ----------------------------------------------------------
    def set_forcing(self, F):
        if F is None:
            self._check(self._L.ns3d_set_forcing(self._h, None, None, None), "set_forcing")
            self._forcing = None
            return
        p = self._fields(F, "forcing")
        self._check(self._L.ns3d_set_forcing(self._h, *p), "ns3d_set_forcing")
        self._forcing = list(F)

    @property
    def forcing_modes(self) -> int:
        return int(self._L.ns3d_forcing_modes(self._h))

    # -- Source/RK_time_step.h --------------------------------------------
    def rk3_ssp(self, U, dt: float, Re: float, nsteps: int = 1):
        """RK3_SSP in place, nsteps times (CUDA-graph replay)."""
        p = self._fields(U, "U")
        self._check(self._L.ns3d_rk3_steps(self._h, *p, dt, Re, int(nsteps)), "ns3d_rk3_steps")
        return U

    def single_time_step(self, U, dt: float, Re: float):
        p = self._fields(U, "U")
        self._check(self._L.ns3d_euler_step(self._h, *p, dt, Re), "ns3d_euler_step")
        return U

    def return_rhs(self, U, Re: float, out=None):
        out = out if out is not None else self.zeros()
        p = self._fields(U, "U")
        q = self._fields(out, "out")
        self._check(self._L.ns3d_rhs(self._h, *p, *q, Re), "ns3d_rhs")
        return out

    def rk3_ssp_uv(self, U, V, dt: float, Re: float, nsteps: int = 1):
        """RK3_SSP_UV: tangent V and base U advanced in place."""
        p = self._fields(U, "U")
        q = self._fields(V, "V")
        self._check(self._L.ns3d_jvp_steps(self._h, *p, *q, dt, Re, int(nsteps)),
                    "ns3d_jvp_steps")
        return U, V

    def rk3_ssp_uv_rhs(self, U, V, Re: float):
        """RK3_SSP_UV_RHS: V <- J(U) V in place."""
        p = self._fields(U, "U")
        q = self._fields(V, "V")
        self._check(self._L.ns3d_linearised_rhs(self._h, *p, *q, Re), "ns3d_linearised_rhs")
        return V

    def single_time_step_uv(self, U, V, dt: float, Re: float):
        """single_time_step_UV: V <- V + dt J(U) V in place (U unchanged)."""
        p = self._fields(U, "U")
        q = self._fields(V, "V")
        self._check(self._L.ns3d_tangent_euler_step(self._h, *p, *q, dt, Re),
                    "ns3d_tangent_euler_step")
        return V

    def single_time_step_iuv_rhs(self, U, V, dt: float, Re: float):
        p = self._fields(U, "U")
        q = self._fields(V, "V")
        self._check(self._L.ns3d_implicit_tangent_step(self._h, *p, *q, dt, Re),
                    "ns3d_implicit_tangent_step")
        return V

    # -- Source/advection_2_3.h -------------------------------------------
    def calculate_convolution_2p3(self, U, out=None):
        out = out if out is not None else self.zeros()
        self._check(self._L.ns3d_convolution(self._h, *self._fields(U, "U"),
                                             *self._fields(out, "out")), "ns3d_convolution")
        return out

    def calculate_convolution_2p3_uv(self, U, V, out=None):
        out = out if out is not None else self.zeros()
        self._check(self._L.ns3d_convolution_uv(self._h, *self._fields(U, "U"),
                                                *self._fields(V, "V"),
                                                *self._fields(out, "out")),
                    "ns3d_convolution_uv")
        return out

    # -- Source/math_support.h: FFTN_Device / iFFTN_Device -----------------
    @property
    def real_shape(self):
        return (self.Nx, self.Ny, self.Nz)

    def fftn(self, x, out=None):
        """FFTN_Device: unnormalised R2C of a real (Nx, Ny, Nz) float64 tensor."""
        t = self._torch
        if (x.dtype != t.float64 or x.device != self.device
                or tuple(x.shape) != self.real_shape or not x.is_contiguous()):
            raise ValueError(f"x: expected contiguous float64 {self.real_shape} on {self.device}")
        out = out if out is not None else t.empty(self.shape, dtype=t.complex128,
                                                  device=self.device)
        self._check(self._L.ns3d_fft_r2c(self._h, _ptr(x), self._fields([out] * 3, "out")[0]),
                    "ns3d_fft_r2c")
        return out

    def ifftn(self, X, out=None, scale: bool = True):
        """iFFTN_Device: C2R of a complex (Nx, Ny, Nz//2+1) tensor, scaled by
        1/(Nx Ny Nz) (scale=False: the two-argument iFFTN_Device, no scale)."""
        t = self._torch
        p = self._fields([X] * 3, "X")[0]
        out = out if out is not None else t.empty(self.real_shape, dtype=t.float64,
                                                  device=self.device)
        if (out.dtype != t.float64 or tuple(out.shape) != self.real_shape
                or not out.is_contiguous() or out.device != self.device):
            raise ValueError("out: expected a contiguous float64 real-space tensor")
        fn = self._L.ns3d_fft_c2r if scale else self._L.ns3d_fft_c2r_unscaled
        self._check(fn(self._h, p, _ptr(out)), "ns3d_fft_c2r")
        return out

    # -- checkpoints (Source/file_operations.cu) -----------------------------
    def save_control_fourier(self, path: str, U):
        """write_control_file_fourier of device fields U."""
        self._check(self._L.ns3d_save_control_fourier(self._h, str(path).encode(),
                                                      *self._fields(U, "U")),
                    "ns3d_save_control_fourier")

    def load_control_fourier(self, path: str, out=None):
        """read_control_fourier into device fields (a coarser file is
        up-sampled the reference's way)."""
        out = out if out is not None else self.zeros()
        self._check(self._L.ns3d_load_control_fourier(self._h, str(path).encode(),
                                                      *self._fields(out, "out")),
                    "ns3d_load_control_fourier")
        return out

    def save_control_file(self, path: str, U):
        """write_control_file of the physical velocity of device fields U."""
        self._check(self._L.ns3d_save_control_file(self._h, str(path).encode(),
                                                   *self._fields(U, "U")),
                    "ns3d_save_control_file")

    def load_control_file(self, path: str, out=None):
        """read_control_file, transformed to spectral device fields."""
        out = out if out is not None else self.zeros()
        self._check(self._L.ns3d_load_control_file(self._h, str(path).encode(),
                                                   *self._fields(out, "out")),
                    "ns3d_load_control_file")
        return out

    # -- Krylov adapters (Source/NS3D_periodic.cu:173-385) ------------------
    @property
    def krylov_length(self) -> int:
        return int(self._L.ns3d_krylov_length(self._h))

    def _vec(self, v, name):
        t = self._torch
        if (v.dtype != t.float64 or v.device != self.device or v.numel() != self.krylov_length
                or not v.is_contiguous()):
            raise ValueError(f"{name}: expected contiguous float64 vector of length "
                             f"{self.krylov_length} on {self.device}")
        return _ptr(v)

    def pack_reduced(self, V, out=None):
        t = self._torch
        out = out if out is not None else t.empty(self.krylov_length, dtype=t.float64,
                                                  device=self.device)
        self._check(self._L.ns3d_pack_reduced(self._h, *self._fields(V, "V"),
                                              self._vec(out, "out")), "ns3d_pack_reduced")
        return out

    def unpack_reduced(self, vec, out=None):
        out = out if out is not None else self.zeros()
        self._check(self._L.ns3d_unpack_reduced(self._h, self._vec(vec, "vec"),
                                                *self._fields(out, "out")),
                    "ns3d_unpack_reduced")
        return out

    def matvec_reduced(self, U, vec_in, Re: float, tau: float = 0.0, out=None):
        """NSCallMatrixVector_reduced (tau <= 0) / _Newton_Globalization (tau > 0)."""
        t = self._torch
        out = out if out is not None else t.empty_like(vec_in)
        self._check(self._L.ns3d_matvec_reduced(self._h, *self._fields(U, "U"),
                                                self._vec(vec_in, "vec_in"),
                                                self._vec(out, "vec_out"), Re, tau),
                    "ns3d_matvec_reduced")
        return out

    # -- diagnostics --------------------------------------------------------
    def diagnostics(self, U):
        """(energy, dissipation, max|div|) as the reference main loop reports them."""
        e, d, dv = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._check(self._L.ns3d_diagnostics(self._h, *self._fields(U, "U"), ctypes.byref(e),
                                             ctypes.byref(d), ctypes.byref(dv)),
                    "ns3d_diagnostics")
        return e.value, d.value, dv.value


    # -- filters, curl and the main loop's record (Source/math_support.cu,
    #    Source/NS3D_periodic.cu:1291-1452, Source/Shapiro_test.cu) ----------
    def _real_fields(self, F: Sequence, name: str):
        t = self._torch
        if len(F) != 3:
            raise ValueError(f"{name}: need 3 components")
        for f in F:
            if (not isinstance(f, t.Tensor) or f.dtype != t.float64 or f.device != self.device
                    or tuple(f.shape) != self.real_shape or not f.is_contiguous()):
                raise ValueError(f"{name}: expected contiguous float64 {self.real_shape} tensors "
                                 f"on {self.device}")
        return [_ptr(f) for f in F]

    def helmholtz_filter(self, U, eps: float, out=None):
        """Helmholz_Fourier_Filter's spectral step: u / (1 + eps^2 |k|^2)."""
        out = out if out is not None else self.zeros()
        self._check(self._L.ns3d_helmholtz_filter(self._h, *self._fields(U, "U"), float(eps),
                                                  *self._fields(out, "out")),
                    "ns3d_helmholtz_filter")
        return out

    def cutoff_filter(self, U, radius: float, out=None):
        """CutOff_Fourier_Filter's spectral step (Mz in its Nz slot)."""
        out = out if out is not None else self.zeros()
        self._check(self._L.ns3d_cutoff_filter(self._h, *self._fields(U, "U"), float(radius),
                                               *self._fields(out, "out")),
                    "ns3d_cutoff_filter")
        return out

    def curl(self, u, out=None):
        """get_curl of physical (Nx, Ny, Nz) float64 fields."""
        t = self._torch
        out = out if out is not None else [t.empty(self.real_shape, dtype=t.float64,
                                                   device=self.device) for _ in range(3)]
        self._check(self._L.ns3d_curl(self._h, *self._real_fields(u, "u"),
                                      *self._real_fields(out, "out")), "ns3d_curl")
        return out

    def record(self, U, total_time: float, Re: float):
        """The 50 columns of one time_dependant.dat line (numpy array)."""
        import numpy as np

        rec = np.zeros(RECORD_COLUMNS)
        rc = self._L.ns3d_record(self._h, *self._fields(U, "U"), float(total_time), float(Re),
                                 rec.ctypes.data)
        if rc == 5:  # non-finite: the record is filled, as main writes it anyway
            return rec
        self._check(rc, "ns3d_record")
        return rec

    def energy_spectrum(self, U):
        """calculate_energy_spectrum's per-bin sums E[n] (numpy array)."""
        import numpy as np

        nb = self.Nx // 2 + self.Ny // 2 + self.Mz
        E = np.zeros(nb)
        self._check(self._L.ns3d_energy_spectrum(self._h, *self._fields(U, "U"), E.ctypes.data,
                                                 nb), "ns3d_energy_spectrum")
        return E

    def write_energy_spectrum(self, path: str, U):
        """Ek.dat of the state, as main writes it at the end of a run."""
        write_energy_spectrum(path, self.Nx, self.Ny, self.Nz, self.energy_spectrum(U))

    def shapiro_state(self, t: float, Re: float, out=None):
        """Shapiro's exact Beltrami solution at time t, spectral."""
        out = out if out is not None else self.zeros()
        self._check(self._L.ns3d_shapiro_state(self._h, float(t), float(Re),
                                               *self._fields(out, "out")), "ns3d_shapiro_state")
        return out

    def shapiro_error(self, U, t: float, Re: float) -> float:
        """Shapiro_test_case: max |u - u_exact(t)| over the grid."""
        e = ctypes.c_double()
        self._check(self._L.ns3d_shapiro_error(self._h, *self._fields(U, "U"), float(t),
                                               float(Re), ctypes.byref(e)), "ns3d_shapiro_error")
        return e.value

    @property
    def precision(self) -> str:
        """"fp64" (the reference's arithmetic) or "fp32" (transforms and
        products in FP32, state and update in FP64)."""
        return "fp32" if self._L.ns3d_get_precision(self._h) == 1 else "fp64"

    @precision.setter
    def precision(self, value: str):
        self._check(self._L.ns3d_set_precision(self._h, _PRECISIONS[value]), "ns3d_set_precision")

    def request_fields(self, Re: float, seed: int):
        """The initial (u, v) of a server request on this (cubic) grid."""
        U, V = self.zeros(), self.zeros()
        self._check(self._L.ns3d_request_fields(self._h, float(Re), int(seed),
                                                *self._fields(U, "U"), *self._fields(V, "V")),
                    "ns3d_request_fields")
        return U, V

    def profile_passes(self, U, dt: float, Re: float, reps: int = 10):
        """Mean ms per launch of (inv_x, inv_y, z, fwd_y, fwd_x), CUDA events."""
        ms = (ctypes.c_double * 5)()
        self._check(self._L.ns3d_profile_passes(self._h, *self._fields(U, "U"), dt, Re,
                                                int(reps), ms), "ns3d_profile_passes")
        return list(ms)

    @property
    def tiles(self):
        """Tile of each pass family (inv_x, inv_y, fwd_y, fwd_x): 0 default,
        1 alternative points per thread, 2 inv_y's bulk-copy (TMA) form
        (y extents from 48), 3 / 4 the default / alternative points per
        thread with the reversed radix schedule (inv_x, inv_y, fwd_y; see
        ns3d_set_tiles)."""
        return _get_tiles(self._L.ns3d_get_tiles, self._h)

    @tiles.setter
    def tiles(self, value):
        t = (ctypes.c_int * 4)(*[int(v) for v in value])
        self._check(self._L.ns3d_set_tiles(self._h, t), "ns3d_set_tiles")

    def autotune(self, reps: int = 20, force: bool = False) -> dict:
        """Times each pass family with each of its tiles and keeps the fastest
        where it beats the default by 2% (ns3d_autotune).  Returns {"tiles":
        [...], "ms": per family {tile: ms} of the tiles timed, None when a
        cached choice was applied}."""
        return _autotune(self._L.ns3d_autotune, self._h, self._check, reps, force,
                         self._L.ns3d_get_tiles)


TILE_FAMILIES = ("inv_x", "inv_y", "fwd_y", "fwd_x")


def _get_tiles(fn, h):
    t = (ctypes.c_int * 4)()
    rc = fn(h, t)
    if rc != 0:
        raise Ns3dError(rc, "get_tiles")
    return list(t)


TILES_PER_FAMILY = 5  # NS3D_TILES_PER_FAMILY


def _autotune(fn, h, check, reps, force, get_fn):
    ms = (ctypes.c_double * (4 * TILES_PER_FAMILY))()  # NS3D_TUNE_TIMES
    check(fn(h, int(reps), int(bool(force)), ms), "autotune")
    times = [{t: ms[TILES_PER_FAMILY * f + t] for t in range(TILES_PER_FAMILY)
              if ms[TILES_PER_FAMILY * f + t] >= 0.0} for f in range(4)]
    timed = any(row for row in times)
    return {"tiles": _get_tiles(get_fn, h), "ms": times if timed else None}


def supported_extent(n: int) -> bool:
    return bool(lib().ns3d_supported_extent(int(n)))


def write_control_fourier(path: str, U):
    """Host form of write_control_file_fourier: U = 3 complex (Nx, Ny, Nz//2+1)
    numpy arrays (Nz taken as 2 (Mz - 1))."""
    import numpy as np

    a = [np.ascontiguousarray(u, dtype=np.complex128) for u in U]
    Nx, Ny, Mz = a[0].shape
    rc = lib().ns3d_write_control_fourier_host(str(path).encode(), Nx, Ny, 2 * (Mz - 1),
                                               *[x.ctypes.data for x in a])
    if rc != 0:
        raise Ns3dError(rc, "ns3d_write_control_fourier_host", str(path))


def read_control_fourier(path: str, Nx: int, Ny: int, Nz: int):
    """Host form of read_control_fourier for an Nx x Ny x Nz grid; returns
    (U, (Nx_file, Ny_file, Mz_file))."""
    import numpy as np

    U = [np.zeros((Nx, Ny, Nz // 2 + 1), dtype=np.complex128) for _ in range(3)]
    ext = [ctypes.c_int(0) for _ in range(3)]
    rc = lib().ns3d_read_control_fourier_host(str(path).encode(), Nx, Ny, Nz,
                                              *[u.ctypes.data for u in U],
                                              *[ctypes.byref(e) for e in ext])
    if rc != 0:
        raise Ns3dError(rc, "ns3d_read_control_fourier_host", str(path))
    return U, tuple(e.value for e in ext)


def write_control_file(path: str, u):
    """Host form of write_control_file: u = 3 real (Nx, Ny, Nz) arrays."""
    import numpy as np

    a = [np.ascontiguousarray(x, dtype=np.float64) for x in u]
    Nx, Ny, Nz = a[0].shape
    rc = lib().ns3d_write_control_file_host(str(path).encode(), Nx, Ny, Nz,
                                            *[x.ctypes.data for x in a])
    if rc != 0:
        raise Ns3dError(rc, "ns3d_write_control_file_host", str(path))


def read_control_file(path: str, Nx: int, Ny: int, Nz: int):
    """Host form of read_control_file."""
    import numpy as np

    u = [np.zeros((Nx, Ny, Nz)) for _ in range(3)]
    rc = lib().ns3d_read_control_file_host(str(path).encode(), Nx, Ny, Nz,
                                           *[x.ctypes.data for x in u])
    if rc != 0:
        raise Ns3dError(rc, "ns3d_read_control_file_host", str(path))
    return u


RECORD_COLUMNS = 50


class TimeSeries:
    """time_dependant.dat of the main loop (ns3d_series_*): one line of 50
    '%le' columns per ``write``.  ``step`` advances the time the reference's
    way (TotalTime += dt twice per step, Source/NS3D_periodic.cu:1355,1374),
    computes the record on the device and writes it."""

    def __init__(self, path: str, total_time: float = 0.0):
        self._L = lib()
        h = ctypes.c_void_p()
        rc = self._L.ns3d_series_open(str(path).encode(), ctypes.byref(h))
        if rc != 0:
            raise Ns3dError(rc, "ns3d_series_open", str(path))
        self._s = h
        self.total_time = float(total_time)

    def write(self, rec):
        import numpy as np

        r = np.ascontiguousarray(rec, dtype=np.float64)
        rc = self._L.ns3d_series_write(self._s, r.ctypes.data, int(r.size))
        if rc != 0:
            raise Ns3dError(rc, "ns3d_series_write", "")

    def step(self, solver: "Solver", U, dt: float, Re: float):
        self.total_time += dt
        self.total_time += dt
        rec = solver.record(U, self.total_time, Re)
        self.write(rec)
        return rec

    def close(self):
        if self._s:
            rc = self._L.ns3d_series_close(self._s)
            self._s = None
            if rc != 0:
                raise Ns3dError(rc, "ns3d_series_close", "")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def write_energy_spectrum(path: str, Nx: int, Ny: int, Nz: int, E):
    """Ek.dat from the per-bin sums E (ns3d_write_energy_spectrum_host)."""
    import numpy as np

    e = np.ascontiguousarray(E, dtype=np.float64)
    if e.size != Nx // 2 + Ny // 2 + Nz // 2 + 1:
        raise ValueError("E must have Nx/2 + Ny/2 + Nz/2 + 1 bins")
    rc = lib().ns3d_write_energy_spectrum_host(str(path).encode(), Nx, Ny, Nz, e.ctypes.data)
    if rc != 0:
        raise Ns3dError(rc, "ns3d_write_energy_spectrum_host", str(path))


class Ensemble:
    """ns3d_ensemble: `batch` independent instances of one grid, each with its
    own dt and Re, advanced together by the launches of one RK3 step.  Fields
    are complex128 tensors of shape (batch, Nx, Ny, Nz//2+1) per component."""

    def __init__(self, batch: int, Nx: int, Ny: int, Nz: int, Lx: float = _PI2,
                 Ly: float = _PI2, Lz: float = _PI2, device=None):
        import torch

        self._torch = torch
        dev = torch.device(device if device is not None else "cuda")
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.batch = int(batch)
        self.Nx, self.Ny, self.Nz = int(Nx), int(Ny), int(Nz)
        self.Mz = self.Nz // 2 + 1
        self._L = lib()
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            torch.cuda.init()
            rc = self._L.ns3d_ensemble_create(self.batch, self.Nx, self.Ny, self.Nz, float(Lx),
                                              float(Ly), float(Lz), ctypes.byref(h))
        if rc != 0:
            raise Ns3dError(rc, "ns3d_ensemble_create")
        self._h = h
        self._forcing = None

    @property
    def shape(self):
        return (self.batch, self.Nx, self.Ny, self.Mz)

    def _check(self, rc: int, where: str):
        if rc != 0:
            detail = self._L.ns3d_ensemble_last_error(self._h)
            raise Ns3dError(rc, where, detail.decode() if detail else "")

    def _fields(self, F, shape, name):
        t = self._torch
        if len(F) != 3:
            raise ValueError(f"{name}: need 3 components")
        for f in F:
            if (not isinstance(f, t.Tensor) or f.dtype != t.complex128 or f.device != self.device
                    or tuple(f.shape) != shape or not f.is_contiguous()):
                raise ValueError(f"{name}: expected contiguous complex128 {shape} tensors")
        return [_ptr(f) for f in F]

    def zeros(self):
        t = self._torch
        return [t.zeros(self.shape, dtype=t.complex128, device=self.device) for _ in range(3)]

    def to_device(self, F):
        t = self._torch
        return [t.as_tensor(f).to(device=self.device, dtype=t.complex128).contiguous() for f in F]

    def set_stream(self, stream):
        raw = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        self._check(self._L.ns3d_ensemble_set_stream(self._h, ctypes.c_void_p(raw)),
                    "ns3d_ensemble_set_stream")

    def set_forcing(self, F):
        """One instance-sized forcing (Nx, Ny, Nz//2+1) shared by all instances."""
        if F is None:
            self._check(self._L.ns3d_ensemble_set_forcing(self._h, None, None, None),
                        "ns3d_ensemble_set_forcing")
            return
        Fd = self.to_device(F)
        p = self._fields(Fd, (self.Nx, self.Ny, self.Mz), "F")
        self._check(self._L.ns3d_ensemble_set_forcing(self._h, *p), "ns3d_ensemble_set_forcing")
        self._forcing = Fd

    def set_precision(self, value: str):
        """"fp64" or "fp32" for every instance (see Solver.precision)."""
        self._check(self._L.ns3d_ensemble_set_precision(self._h, _PRECISIONS[value]),
                    "ns3d_ensemble_set_precision")

    @property
    def tiles(self):
        """Pass tiles of the batch (see Solver.tiles)."""
        return _get_tiles(self._L.ns3d_ensemble_get_tiles, self._h)

    @tiles.setter
    def tiles(self, value):
        t = (ctypes.c_int * 4)(*[int(v) for v in value])
        self._check(self._L.ns3d_ensemble_set_tiles(self._h, t), "ns3d_ensemble_set_tiles")

    def autotune(self, reps: int = 20, force: bool = False) -> dict:
        """Solver.autotune for the ensemble's batch (ns3d_ensemble_autotune)."""
        return _autotune(self._L.ns3d_ensemble_autotune, self._h, self._check, reps, force,
                         self._L.ns3d_ensemble_get_tiles)

    def set_params(self, dt, Re):
        import numpy as np

        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, np.float64), (self.batch,)))
        r = np.ascontiguousarray(np.broadcast_to(np.asarray(Re, np.float64), (self.batch,)))
        self._check(self._L.ns3d_ensemble_set_params(self._h, d.ctypes.data, r.ctypes.data),
                    "ns3d_ensemble_set_params")

    def rk3_steps(self, U, nsteps: int = 1):
        self._check(self._L.ns3d_ensemble_rk3_steps(self._h, *self._fields(U, self.shape, "U"),
                                                    int(nsteps)), "ns3d_ensemble_rk3_steps")
        return U

    def diagnostics(self, U):
        """(energy, dissipation) per instance; an instance whose values are
        not finite has diverged (the call still returns)."""
        import numpy as np

        e = np.zeros(self.batch)
        d = np.zeros(self.batch)
        rc = self._L.ns3d_ensemble_diagnostics(self._h, *self._fields(U, self.shape, "U"),
                                               e.ctypes.data, d.ctypes.data)
        if rc != 5:  # non-finite: the arrays are filled, NaN/Inf marks diverged instances
            self._check(rc, "ns3d_ensemble_diagnostics")
        return e, d

    @property
    def device_bytes(self) -> int:
        return int(self._L.ns3d_ensemble_device_bytes(self._h))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.ns3d_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def request_steps(N: int, Re: float, T: float) -> int:
    """JVP steps of a server request: ceil(T / dt), dt = 0.3 (2 pi/N) / (Re/16)."""
    return int(lib().ns3d_request_steps(int(N), float(Re), float(T)))


class Server:
    """ns3d_server: tangent-integration requests served with continuous
    batching, one batched slot pool per grid N (see include/ns3d.h)."""

    def __init__(self, Ns, capacity=None, hbm_fraction: float = 0.0, device=None):
        """capacity: slots per grid (at most, with hbm_fraction in (0, 1));
        without it, hbm_fraction (default 0.5) of the free device memory sets
        them."""
        import torch

        if capacity is None and not 0.0 < hbm_fraction < 1.0:
            hbm_fraction = 0.5
        self._L = lib()
        dev = torch.device(device if device is not None else "cuda")
        Ns = [int(n) for n in Ns]
        arr = (ctypes.c_int * len(Ns))(*Ns)
        cap = (ctypes.c_int * len(Ns))(*[int(c) for c in capacity]) if capacity else None
        h = ctypes.c_void_p()
        with torch.cuda.device(dev):
            torch.cuda.init()
            rc = self._L.ns3d_server_create(arr, len(Ns), cap, float(hbm_fraction),
                                            ctypes.byref(h))
        if rc != 0:
            raise Ns3dError(rc, "ns3d_server_create")
        self._h = h
        self.Ns = Ns
        self._held = {}     # tensors of field requests not yet done
        self._forcing = {}  # forcing tensors set per grid

    def _check(self, rc, where):
        if rc != 0:
            d = self._L.ns3d_server_last_error(self._h)
            raise Ns3dError(rc, where, d.decode() if d else "")

    def capacity(self, N: int) -> int:
        c = ctypes.c_int()
        self._check(self._L.ns3d_server_capacity(self._h, int(N), ctypes.byref(c)),
                    "ns3d_server_capacity")
        return c.value

    def set_precision(self, value: str):
        """"fp64" or "fp32" for every grid (between runs)."""
        self._check(self._L.ns3d_server_set_precision(self._h, _PRECISIONS[value]),
                    "ns3d_server_set_precision")

    def autotune(self, reps: int = 10):
        """Tile autotuner for every grid at its slot count (between runs)."""
        self._check(self._L.ns3d_server_autotune(self._h, int(reps)), "ns3d_server_autotune")

    def instance_steps(self, N: int) -> int:
        """JVP steps grid N has run so far, summed over its slots."""
        c = ctypes.c_longlong()
        self._check(self._L.ns3d_server_stats(self._h, int(N), ctypes.byref(c)),
                    "ns3d_server_stats")
        return c.value

    def submit(self, requests):
        """requests: iterable of dicts or tuples (N, Re, T, seed[, arrival[, keep]]),
        in arrival order.  Returns the first id."""
        rs = []
        for r in requests:
            if isinstance(r, dict):
                rs.append(Request(int(r["N"]), float(r["Re"]), float(r["T"]), int(r["seed"]),
                                  float(r.get("arrival", 0.0)), int(r.get("keep", 0))))
            else:
                rs.append(Request(int(r[0]), float(r[1]), float(r[2]), int(r[3]),
                                  float(r[4]) if len(r) > 4 else 0.0,
                                  int(r[5]) if len(r) > 5 else 0))
        arr = (Request * max(len(rs), 1))(*rs)
        first = ctypes.c_longlong()
        self._check(self._L.ns3d_server_submit(self._h, arr, len(rs), ctypes.byref(first)),
                    "ns3d_server_submit")
        return first.value

    def submit_fields(self, requests):
        """Requests that carry their own fields (ns3d_field_request), in
        arrival order: dicts with N, Re, dt, steps, U and V (three CUDA
        complex128 tensors each, [N, N, N/2+1]), V_out (default V: v(T) is
        written back in place), U_out (default None: u(T) is not returned)
        and arrival (default -1: now).  The tensors stay referenced until the
        request is done.  Returns the first id."""
        rs, keep = [], []
        for r in requests:
            N = int(r["N"])
            U, V = r["U"], r["V"]
            Vo = r.get("V_out", V)
            Uo = r.get("U_out")
            for F in (U, V, Vo) + ((Uo,) if Uo is not None else ()):
                self._field_check(F, N)
            q = FieldRequest()
            q.N, q.Re, q.dt, q.steps = N, float(r["Re"]), float(r["dt"]), int(r["steps"])
            for c in range(3):
                q.u_in[c] = U[c].data_ptr()
                q.v_in[c] = V[c].data_ptr()
                q.v_out[c] = Vo[c].data_ptr()
                q.u_out[c] = Uo[c].data_ptr() if Uo is not None else None
            q.arrival = float(r.get("arrival", -1.0))
            rs.append(q)
            keep.append((U, V, Vo, Uo))
        arr = (FieldRequest * max(len(rs), 1))(*rs)
        first = ctypes.c_longlong()
        self._check(self._L.ns3d_server_submit_fields(self._h, arr, len(rs),
                                                      ctypes.byref(first)),
                    "ns3d_server_submit_fields")
        for i, k in enumerate(keep):
            self._held[first.value + i] = k
        return first.value

    @staticmethod
    def _field_check(F, N):
        import torch

        Mz = N // 2 + 1
        if len(F) != 3 or any(f.dtype != torch.complex128 or not f.is_contiguous() or
                              tuple(f.shape) != (N, N, Mz) for f in F):
            raise ValueError(f"fields must be 3 contiguous complex128 tensors of shape "
                             f"({N}, {N}, {Mz})")

    def set_forcing(self, N: int, F):
        """Forcing of grid N's base flow (three CUDA tensors), between runs."""
        self._field_check(F, int(N))
        self._check(self._L.ns3d_server_set_forcing(self._h, int(N),
                                                    *[f.data_ptr() for f in F]),
                    "ns3d_server_set_forcing")
        self._forcing[int(N)] = F

    def cancel(self, rid: int):
        """ns3d_server_cancel (may be called while run() runs on another thread)."""
        self._check(self._L.ns3d_server_cancel(self._h, int(rid)), "ns3d_server_cancel")

    def run(self, max_seconds: float = 1e30) -> int:
        n = ctypes.c_int()
        self._check(self._L.ns3d_server_run(self._h, float(max_seconds), ctypes.byref(n)),
                    "ns3d_server_run")
        self._release()
        return n.value

    def run_until(self, rid: int, max_seconds: float = 1e30) -> int:
        """Runs until request rid is done (ns3d_server_run_until)."""
        n = ctypes.c_int()
        self._check(self._L.ns3d_server_run_until(self._h, int(rid), float(max_seconds),
                                                  ctypes.byref(n)),
                    "ns3d_server_run_until")
        self._release()
        return n.value

    def _release(self):
        if self._held:
            done = {r["id"] for r in self.results() if r["status"] != -1}
            for rid in [k for k in self._held if k in done]:
                del self._held[rid]

    def results(self):
        n = ctypes.c_int()
        self._check(self._L.ns3d_server_results(self._h, None, 0, ctypes.byref(n)),
                    "ns3d_server_results")
        arr = (Result * max(n.value, 1))()
        self._check(self._L.ns3d_server_results(self._h, arr, n.value, ctypes.byref(n)),
                    "ns3d_server_results")
        return [{f: getattr(arr[i], f) for f, _ in Result._fields_} for i in range(n.value)]

    def result_field(self, rid: int, N: int):
        """v(T) of a request submitted with keep = 1 (host numpy arrays)."""
        import numpy as np

        Mz = N // 2 + 1
        v = [np.zeros((N, N, Mz), np.complex128) for _ in range(3)]
        self._check(self._L.ns3d_server_result_field(self._h, int(rid),
                                                     *[x.ctypes.data for x in v]),
                    "ns3d_server_result_field")
        return v

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.ns3d_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
