"""Drop-in at the link level: the harness that drives the reference's own build
(oracle/ref_harness.cu, written against the reference headers and calling
RK3_SSP, return_RHS, calculate_convolution_2p3[_UV], RK3_SSP_UV[_RHS],
single_time_step[_iUV_RHS], FFTN_Device / iFFTN_Device, Image_to_Domain,
get_kinetic_energy / get_dissipation and the host table builders exactly as
main() does) is linked against this project's reference-signature layer
(libns3d_compat.so) instead of the reference's objects, and must reproduce
the reference's golden outputs.  Tolerance: relative L2 <= 1e-12.
"""
import os

import numpy as np
import pytest

from oracle import ns3d_oracle as O
from oracle import ref_lib

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


@pytest.fixture(scope="module")
def torch():
    import torch as t

    if not t.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return t


@pytest.fixture(scope="module")
def compat_lib():
    if not os.path.exists(ref_lib.COMPAT_LIB_PATH):
        pytest.fail("oracle/_ref/libns3d_ref_compat.so is missing (make -C oracle)")
    return ref_lib.COMPAT_LIB_PATH


@pytest.mark.parametrize("case", ["iso16", "aniso16x8x24"])
def test_reference_harness_on_compat_layer_matches_golden(torch, golden, compat_lib, case):
    d = golden[case]
    Nx, Ny, Nz = int(d["Nx"]), int(d["Ny"]), int(d["Nz"])
    Re, dt = float(d["Re"]), float(d["dt"])
    Uo, Vo, Ug, F = list(d["U_odd"]), list(d["V_odd"]), list(d["U_gen"]), list(d["F"])
    with ref_lib.RefSolver(Nx, Ny, Nz, float(d["Lx"]), float(d["Ly"]), float(d["Lz"]),
                           lib_path=compat_lib) as R:
        assert _rel(R.c2r(d["X_nonherm"]), d["c2r_nonherm"]) < TOL
        R.set_f(F)
        R.set_u(Uo)
        assert _rel(R.conv(), d["conv_odd"]) < TOL
        R.set_u(Ug)
        assert _rel(R.conv(), d["conv_gen"]) < TOL
        R.set_u(Uo)
        R.set_v(Vo)
        assert _rel(R.conv_uv(), d["conv_uv"]) < TOL
        R.set_u(Uo)
        assert _rel(R.rhs(Re), d["rhs_odd"]) < TOL
        R.set_u(Uo)
        R.euler(dt, Re)
        assert _rel(R.get_u(), d["euler_odd"]) < TOL
        R.set_u(Uo)
        R.rk3(1, dt, Re)
        assert _rel(R.get_u(), d["rk3x1_odd"]) < TOL
        R.set_u(Uo)
        R.rk3(5, dt, Re)
        assert _rel(R.get_u(), d["rk3x5_odd"]) < TOL
        R.set_u(Ug)
        R.rk3(1, dt, Re)
        assert _rel(R.get_u(), d["rk3x1_gen"]) < TOL
        R.set_u(Uo)
        R.set_v(Vo)
        R.jvp(1, dt, Re)
        assert _rel(R.get_u(), d["jvp_u"]) < TOL
        assert _rel(R.get_v(), d["jvp_v"]) < TOL
        R.set_u(Uo)
        R.set_v(Vo)
        R.linrhs(dt, Re)
        assert _rel(R.get_v(), d["linrhs_v"]) < TOL
        R.set_u(Uo)
        R.set_v(Vo)
        R.iuv(dt, Re)
        assert _rel(R.get_v(), d["iuv_v"]) < TOL
        R.set_u(Uo)
        e, diss = R.diag()
        assert abs(e / d["diag_odd"][0] - 1.0) < 1e-12
        assert abs(diss / d["diag_odd"][1] - 1.0) < 1e-12
        # R2C through FFTN_Device (no grid arguments: the grid in use)
        g = O.Grid(Nx, Ny, Nz, float(d["Lx"]), float(d["Ly"]), float(d["Lz"]))
        x = np.random.default_rng(5).standard_normal((Nx, Ny, Nz))
        assert _rel(R.r2c(x), O.r2c(g, x)) < TOL


def test_compat_forcing_pointer_cache(torch, golden, compat_lib):
    """New forcing values under the same pointers are picked up after
    ns3d_compat_forcing_changed; new pointers are picked up by themselves."""
    d = golden["iso16"]
    Re, dt = float(d["Re"]), float(d["dt"])
    g = O.Grid(16, 16, 16)
    Uo = list(d["U_odd"])
    F2 = [2.0 * f for f in d["F"]]
    with ref_lib.RefSolver(16, 16, 16, lib_path=compat_lib) as R:
        R.set_f(list(d["F"]))
        R.set_u(Uo)
        R.rk3(1, dt, Re)
        # same device arrays, new contents: the harness rewrites S.f in place
        R.set_f(F2)
        import ctypes

        lib = ctypes.CDLL(os.path.join(os.path.dirname(ref_lib.COMPAT_LIB_PATH), "..", "..",
                                       "ns3dperiodic_b200", "libns3d_compat.so"))
        getattr(lib, "_Z27ns3d_compat_forcing_changedv")()
        R.set_u(Uo)
        R.rk3(1, dt, Re)
        got = R.get_u()
    assert _rel(got, O.rk3_ssp(g, Uo, F2, dt, Re)) < TOL
