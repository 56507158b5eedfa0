"""ctypes binding of libns3d_b200.so (the C ABI declared in include/ns3d.h).

The CUDA library is the product path; there is no fallback.  If the shared
library is missing or fails to load, importing any compute entry point
raises :class:`Ns3dLibraryError`.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libns3d_b200.so")

STATUS = {
    0: "ok",
    1: "bad argument",
    2: "unsupported grid extent",
    3: "out of device memory",
    4: "CUDA error",
    5: "non-finite value",
    6: "device wait timed out",
    7: "inner linear solve did not converge",
    8: "request cancelled",
}

# every symbol include/ns3d.h declares
EXPORTS = (
    "ns3d_create", "ns3d_destroy", "ns3d_supported_extent", "ns3d_selftest_bounded_wait", "ns3d_set_stream",
    "ns3d_synchronize", "ns3d_last_error", "ns3d_status_string", "ns3d_device_bytes",
    "ns3d_set_forcing", "ns3d_forcing_modes", "ns3d_rk3_step", "ns3d_rk3_steps",
    "ns3d_euler_step", "ns3d_rhs", "ns3d_convolution", "ns3d_convolution_uv",
    "ns3d_jvp_step", "ns3d_jvp_steps", "ns3d_linearised_rhs", "ns3d_implicit_tangent_step",
    "ns3d_krylov_length", "ns3d_pack_reduced", "ns3d_pack_reduced_shifted",
    "ns3d_unpack_reduced", "ns3d_matvec_reduced",
    "ns3d_diagnostics", "ns3d_profile_passes", "ns3d_mask_cutoff", "ns3d_twiddles",
    "ns3d_save_control_fourier", "ns3d_load_control_fourier", "ns3d_save_control_file",
    "ns3d_load_control_file", "ns3d_write_control_fourier_host", "ns3d_read_control_fourier_host",
    "ns3d_write_control_file_host", "ns3d_read_control_file_host",
    "ns3d_convolution_noalloc", "ns3d_fft_r2c", "ns3d_fft_c2r", "ns3d_fft_c2r_unscaled",
    "ns3d_tangent_euler_step",
    "ns3d_krylov_create", "ns3d_krylov_destroy", "ns3d_krylov_set_stream",
    "ns3d_krylov_last_error", "ns3d_arnoldi", "ns3d_krylov_stats", "ns3d_qr_shifts",
    "ns3d_ira_restart", "ns3d_krylov_profile", "ns3d_krylov_combine", "ns3d_bicgstabl", "ns3d_newton",
    "ns3d_map_rhs", "ns3d_map_linearised", "ns3d_map_exponential", "ns3d_map_laplace1d",
    "ns3d_map_exponential_shifted", "ns3d_map_exponential_rotated", "ns3d_map_exponent_invert",
    "ns3d_map_rotated_exponent_invert",
    "ns3d_helmholtz_filter", "ns3d_cutoff_filter", "ns3d_curl", "ns3d_record",
    "ns3d_energy_spectrum", "ns3d_shapiro_state", "ns3d_shapiro_error_physical",
    "ns3d_shapiro_error", "ns3d_series_open", "ns3d_series_write", "ns3d_series_close",
    "ns3d_write_energy_spectrum_host",
    "ns3d_ensemble_create", "ns3d_ensemble_destroy", "ns3d_ensemble_set_stream",
    "ns3d_ensemble_last_error", "ns3d_ensemble_device_bytes", "ns3d_ensemble_set_forcing",
    "ns3d_ensemble_set_params", "ns3d_ensemble_rk3_steps", "ns3d_ensemble_diagnostics",
    "ns3d_set_precision", "ns3d_get_precision", "ns3d_ensemble_set_precision",
    "ns3d_get_tiles", "ns3d_set_tiles", "ns3d_autotune", "ns3d_ensemble_autotune",
    "ns3d_ensemble_get_tiles", "ns3d_ensemble_set_tiles", "ns3d_server_autotune",
    "ns3d_server_create", "ns3d_server_destroy", "ns3d_server_last_error",
    "ns3d_server_capacity", "ns3d_server_stats", "ns3d_server_set_precision", "ns3d_server_submit", "ns3d_server_run", "ns3d_server_results",
    "ns3d_server_result_field", "ns3d_request_fields", "ns3d_request_steps",
    "ns3d_server_submit_fields", "ns3d_server_set_forcing", "ns3d_server_cancel",
    "ns3d_server_run_until", "ns3d_map_exponential_served",
)

class Request(ctypes.Structure):
    """ns3d_request of include/ns3d.h."""
    _fields_ = [("N", ctypes.c_int), ("Re", ctypes.c_double), ("T", ctypes.c_double),
                ("seed", ctypes.c_ulonglong), ("arrival", ctypes.c_double),
                ("keep", ctypes.c_int)]


class Result(ctypes.Structure):
    """ns3d_result of include/ns3d.h."""
    _fields_ = [("id", ctypes.c_longlong), ("N", ctypes.c_int), ("Re", ctypes.c_double),
                ("T", ctypes.c_double), ("steps", ctypes.c_int), ("arrival", ctypes.c_double),
                ("admitted", ctypes.c_double), ("done", ctypes.c_double),
                ("v_norm", ctypes.c_double), ("status", ctypes.c_int)]


class FieldRequest(ctypes.Structure):
    """ns3d_field_request of include/ns3d.h."""
    _fields_ = [("N", ctypes.c_int), ("Re", ctypes.c_double), ("dt", ctypes.c_double),
                ("steps", ctypes.c_int), ("u_in", ctypes.c_void_p * 3),
                ("v_in", ctypes.c_void_p * 3), ("u_out", ctypes.c_void_p * 3),
                ("v_out", ctypes.c_void_p * 3), ("arrival", ctypes.c_double)]


# the matrix-vector callback type of ns3d_arnoldi: void (*)(void*, void*, void*)
MAP_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p)


class MapContext(ctypes.Structure):
    """ns3d_map_context of include/ns3d.h."""
    _fields_ = [("solver", ctypes.c_void_p),
                ("ux", ctypes.c_void_p), ("uy", ctypes.c_void_p), ("uz", ctypes.c_void_p),
                ("vx", ctypes.c_void_p), ("vy", ctypes.c_void_p), ("vz", ctypes.c_void_p),
                ("dt", ctypes.c_double), ("Re", ctypes.c_double), ("tau", ctypes.c_double),
                ("steps", ctypes.c_int), ("status", ctypes.c_int)]


class ServedMapContext(ctypes.Structure):
    """ns3d_served_map_context of include/ns3d.h."""
    _fields_ = [("map", MapContext), ("server", ctypes.c_void_p),
                ("requests", ctypes.c_longlong)]


class ShiftInvertContext(ctypes.Structure):
    """ns3d_shift_invert_context of include/ns3d.h."""
    _fields_ = [("map", MapContext), ("shift_real", ctypes.c_double),
                ("rotate_angle", ctypes.c_double), ("L", ctypes.c_int), ("tol", ctypes.c_double),
                ("max_iter", ctypes.c_int), ("warm_start", ctypes.c_int),
                ("inner", ctypes.c_void_p), ("last_flag", ctypes.c_int),
                ("last_iter", ctypes.c_int), ("last_tol", ctypes.c_double),
                ("solves", ctypes.c_longlong), ("inner_iter", ctypes.c_longlong)]


class LaplaceContext(ctypes.Structure):
    """ns3d_laplace_context of include/ns3d.h."""
    _fields_ = [("n", ctypes.c_int64), ("stream", ctypes.c_void_p), ("status", ctypes.c_int)]


class Ns3dLibraryError(RuntimeError):
    pass


class Ns3dError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        msg = f"{where}: {STATUS.get(status, status)}"
        if detail:
            msg += f" ({detail})"
        super().__init__(msg)


_lib = None

c_int, c_double, c_void_p, c_int64, c_size_t = (ctypes.c_int, ctypes.c_double, ctypes.c_void_p,
                                                ctypes.c_int64, ctypes.c_size_t)
_P = c_void_p


def _sig(lib):
    S = {
        "ns3d_create": ([c_int, c_int, c_int, c_double, c_double, c_double,
                         ctypes.POINTER(c_void_p)], c_int),
        "ns3d_destroy": ([_P], c_int),
        "ns3d_supported_extent": ([c_int], c_int),
        "ns3d_selftest_bounded_wait": ([_P], c_int),
        "ns3d_set_stream": ([_P, _P], c_int),
        "ns3d_synchronize": ([_P], c_int),
        "ns3d_last_error": ([_P], ctypes.c_char_p),
        "ns3d_status_string": ([c_int], ctypes.c_char_p),
        "ns3d_device_bytes": ([_P], c_size_t),
        "ns3d_set_forcing": ([_P, _P, _P, _P], c_int),
        "ns3d_forcing_modes": ([_P], c_int),
        "ns3d_rk3_step": ([_P, _P, _P, _P, c_double, c_double], c_int),
        "ns3d_rk3_steps": ([_P, _P, _P, _P, c_double, c_double, c_int], c_int),
        "ns3d_euler_step": ([_P, _P, _P, _P, c_double, c_double], c_int),
        "ns3d_rhs": ([_P] + [_P] * 6 + [c_double], c_int),
        "ns3d_convolution": ([_P] + [_P] * 6, c_int),
        "ns3d_convolution_uv": ([_P] + [_P] * 9, c_int),
        "ns3d_jvp_step": ([_P] + [_P] * 6 + [c_double, c_double], c_int),
        "ns3d_jvp_steps": ([_P] + [_P] * 6 + [c_double, c_double, c_int], c_int),
        "ns3d_linearised_rhs": ([_P] + [_P] * 6 + [c_double], c_int),
        "ns3d_implicit_tangent_step": ([_P] + [_P] * 6 + [c_double, c_double], c_int),
        "ns3d_krylov_length": ([_P], c_int64),
        "ns3d_pack_reduced": ([_P] + [_P] * 3 + [_P], c_int),
        "ns3d_pack_reduced_shifted": ([_P] + [_P] * 3 + [_P, c_double, _P, c_double, _P], c_int),
        "ns3d_unpack_reduced": ([_P, _P] + [_P] * 3, c_int),
        "ns3d_matvec_reduced": ([_P] + [_P] * 3 + [_P, _P, c_double, c_double], c_int),
        "ns3d_diagnostics": ([_P] + [_P] * 3 + [_P, _P, _P], c_int),
        "ns3d_profile_passes": ([_P] + [_P] * 3 + [c_double, c_double, c_int, _P], c_int),
        "ns3d_mask_cutoff": ([c_int, c_int, c_int, c_double, c_double, c_double, _P], c_int),
        "ns3d_twiddles": ([c_int, _P], c_int),
        "ns3d_convolution_noalloc": ([c_int, c_int, c_int, c_double, c_double, c_double]
                                     + [_P] * 6 + [_P], c_int),
        "ns3d_fft_r2c": ([_P, _P, _P], c_int),
        "ns3d_save_control_fourier": ([_P, ctypes.c_char_p, _P, _P, _P], c_int),
        "ns3d_load_control_fourier": ([_P, ctypes.c_char_p, _P, _P, _P], c_int),
        "ns3d_save_control_file": ([_P, ctypes.c_char_p, _P, _P, _P], c_int),
        "ns3d_load_control_file": ([_P, ctypes.c_char_p, _P, _P, _P], c_int),
        "ns3d_write_control_fourier_host": ([ctypes.c_char_p, c_int, c_int, c_int, _P, _P, _P],
                                            c_int),
        "ns3d_read_control_fourier_host": ([ctypes.c_char_p, c_int, c_int, c_int, _P, _P, _P,
                                            _P, _P, _P], c_int),
        "ns3d_write_control_file_host": ([ctypes.c_char_p, c_int, c_int, c_int, _P, _P, _P],
                                         c_int),
        "ns3d_read_control_file_host": ([ctypes.c_char_p, c_int, c_int, c_int, _P, _P, _P],
                                        c_int),
        "ns3d_fft_c2r": ([_P, _P, _P], c_int),
        "ns3d_fft_c2r_unscaled": ([_P, _P, _P], c_int),
        "ns3d_tangent_euler_step": ([_P] + [_P] * 6 + [c_double, c_double], c_int),
        "ns3d_krylov_create": ([c_int64, c_int, ctypes.POINTER(c_void_p)], c_int),
        "ns3d_krylov_destroy": ([_P], c_int),
        "ns3d_krylov_set_stream": ([_P, _P], c_int),
        "ns3d_krylov_last_error": ([_P], ctypes.c_char_p),
        "ns3d_arnoldi": ([_P, _P, _P, _P, _P, _P, c_int, c_int], c_int),
        "ns3d_krylov_stats": ([_P, _P, _P, _P], c_int),
        "ns3d_qr_shifts": ([c_int, c_int, _P, _P, _P, _P, _P], c_int),
        "ns3d_ira_restart": ([_P, _P, _P, _P, _P, c_int, c_int, _P], c_int),
        "ns3d_krylov_profile": ([_P, _P, c_int, _P, c_int, _P], c_int),
        "ns3d_krylov_combine": ([_P, _P, c_int, _P, c_int, _P], c_int),
        "ns3d_bicgstabl": ([_P, c_int, _P, _P, _P, _P, _P, _P, _P], c_int),
        "ns3d_newton": ([_P, _P, _P, _P, _P, _P, _P, _P, c_double, c_int, _P, _P], c_int),
        "ns3d_map_rhs": ([_P, _P, _P], None),
        "ns3d_map_linearised": ([_P, _P, _P], None),
        "ns3d_map_exponential": ([_P, _P, _P], None),
        "ns3d_map_laplace1d": ([_P, _P, _P], None),
        "ns3d_map_exponential_shifted": ([_P, _P, _P], None),
        "ns3d_map_exponential_rotated": ([_P, _P, _P], None),
        "ns3d_map_exponent_invert": ([_P, _P, _P], None),
        "ns3d_map_rotated_exponent_invert": ([_P, _P, _P], None),
        "ns3d_helmholtz_filter": ([_P, _P, _P, _P, c_double, _P, _P, _P], c_int),
        "ns3d_cutoff_filter": ([_P, _P, _P, _P, c_double, _P, _P, _P], c_int),
        "ns3d_curl": ([_P] + [_P] * 6, c_int),
        "ns3d_record": ([_P, _P, _P, _P, c_double, c_double, _P], c_int),
        "ns3d_energy_spectrum": ([_P, _P, _P, _P, _P, c_int], c_int),
        "ns3d_shapiro_state": ([_P, c_double, c_double, _P, _P, _P], c_int),
        "ns3d_shapiro_error_physical": ([_P, _P, _P, _P, c_double, c_double, _P], c_int),
        "ns3d_shapiro_error": ([_P, _P, _P, _P, c_double, c_double, _P], c_int),
        "ns3d_series_open": ([ctypes.c_char_p, ctypes.POINTER(c_void_p)], c_int),
        "ns3d_series_write": ([_P, _P, c_int], c_int),
        "ns3d_series_close": ([_P], c_int),
        "ns3d_write_energy_spectrum_host": ([ctypes.c_char_p, c_int, c_int, c_int, _P], c_int),
        "ns3d_ensemble_create": ([c_int, c_int, c_int, c_int, c_double, c_double, c_double,
                                  ctypes.POINTER(c_void_p)], c_int),
        "ns3d_ensemble_destroy": ([_P], c_int),
        "ns3d_ensemble_set_stream": ([_P, _P], c_int),
        "ns3d_ensemble_last_error": ([_P], ctypes.c_char_p),
        "ns3d_ensemble_device_bytes": ([_P], ctypes.c_size_t),
        "ns3d_ensemble_set_forcing": ([_P, _P, _P, _P], c_int),
        "ns3d_ensemble_set_params": ([_P, _P, _P], c_int),
        "ns3d_ensemble_rk3_steps": ([_P, _P, _P, _P, c_int], c_int),
        "ns3d_ensemble_diagnostics": ([_P, _P, _P, _P, _P, _P], c_int),
        "ns3d_set_precision": ([_P, c_int], c_int),
        "ns3d_get_precision": ([_P], c_int),
        "ns3d_ensemble_set_precision": ([_P, c_int], c_int),
        "ns3d_get_tiles": ([_P, _P], c_int),
        "ns3d_set_tiles": ([_P, _P], c_int),
        "ns3d_autotune": ([_P, c_int, c_int, _P], c_int),
        "ns3d_ensemble_autotune": ([_P, c_int, c_int, _P], c_int),
        "ns3d_ensemble_get_tiles": ([_P, _P], c_int),
        "ns3d_ensemble_set_tiles": ([_P, _P], c_int),
        "ns3d_server_autotune": ([_P, c_int], c_int),
        "ns3d_server_create": ([_P, c_int, _P, c_double, ctypes.POINTER(c_void_p)], c_int),
        "ns3d_server_destroy": ([_P], c_int),
        "ns3d_server_last_error": ([_P], ctypes.c_char_p),
        "ns3d_server_capacity": ([_P, c_int, _P], c_int),
        "ns3d_server_stats": ([_P, c_int, _P], c_int),
        "ns3d_server_set_precision": ([_P, c_int], c_int),
        "ns3d_server_submit": ([_P, _P, c_int, _P], c_int),
        "ns3d_server_run": ([_P, c_double, _P], c_int),
        "ns3d_server_results": ([_P, _P, c_int, _P], c_int),
        "ns3d_server_result_field": ([_P, ctypes.c_longlong, _P, _P, _P], c_int),
        "ns3d_request_fields": ([_P, c_double, ctypes.c_ulonglong] + [_P] * 6, c_int),
        "ns3d_request_steps": ([c_int, c_double, c_double], c_int),
        "ns3d_server_submit_fields": ([_P, _P, c_int, _P], c_int),
        "ns3d_server_set_forcing": ([_P, c_int, _P, _P, _P], c_int),
        "ns3d_server_cancel": ([_P, ctypes.c_longlong], c_int),
        "ns3d_server_run_until": ([_P, ctypes.c_longlong, c_double, _P], c_int),
        "ns3d_map_exponential_served": ([_P, _P, _P], None),
    }
    for name, (args, res) in S.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res


def lib():
    """The loaded CUDA library (raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise Ns3dLibraryError(
                f"{LIB_PATH} is missing: build it with `python -m ns3dperiodic_b200.build`")
        try:
            l = ctypes.CDLL(LIB_PATH)
        except OSError as e:  # pragma: no cover
            raise Ns3dLibraryError(f"cannot load {LIB_PATH}: {e}") from e
        _sig(l)
        _lib = l
    return _lib
