"""The C++ / OpenMP restatement of the RK3 step (oracle/cpu_rk3.cpp, the CPU
baseline) against the reference's golden vectors and the numpy oracle.
Tolerance: relative L2 <= 1e-12.  No GPU needed."""
import math
import os
import subprocess

import pytest

from oracle import cpu_lib
from oracle import ns3d_oracle as O

TOL = 1e-12


@pytest.fixture(scope="module")
def port():
    if not cpu_lib.available():
        # the oracle folder itself: _cpu/ does not exist before the first build
        subprocess.run(["make", "-C", os.path.dirname(os.path.dirname(cpu_lib.LIB_PATH)), "cpu"],
                       check=True, capture_output=True)
    return cpu_lib


@pytest.mark.parametrize("case", ["iso16", "aniso16x8x24"])
def test_port_matches_reference_golden(port, golden, case):
    d = golden[case]
    Nx, Ny, Nz = int(d["Nx"]), int(d["Ny"]), int(d["Nz"])
    with port.CpuRK3(Nx, Ny, Nz, float(d["Lx"]), float(d["Ly"]), float(d["Lz"])) as C:
        C.set_forcing(list(d["F"]))
        for src, key in (("U_odd", "conv_odd"), ("U_gen", "conv_gen")):
            assert O.rel_l2(C.convolution(list(d[src])), list(d[key])) < TOL
        for src, n, key in (("U_odd", 1, "rk3x1_odd"), ("U_odd", 5, "rk3x5_odd"),
                            ("U_gen", 1, "rk3x1_gen")):
            got = C.rk3_ssp(list(d[src]), float(d["dt"]), float(d["Re"]), n)
            assert O.rel_l2(got, list(d[key])) < TOL, key


@pytest.mark.parametrize("shape", [(24, 32, 48), (48, 12, 16)])
def test_port_matches_oracle_on_3_2k_grids(port, shape):
    g = O.Grid(*shape, 2 * math.pi, 3.0, 5.0)
    U, F = O.kolmogorov_state(g, 80.0, 3, rel_amp=0.2)
    with port.CpuRK3(*shape, 2 * math.pi, 3.0, 5.0) as C:
        C.set_forcing(F)
        got = C.rk3_ssp(U, 2e-3, 80.0, 2)
    ref = O.rk3_ssp(g, O.rk3_ssp(g, U, F, 2e-3, 80.0), F, 2e-3, 80.0)
    assert O.rel_l2(got, ref) < TOL
