"""The oracle against golden vectors of the reference's own CUDA build.

tests/golden/*.npz were produced by tests/golden/make_golden.py, which runs
the unmodified reference sources (oracle/_ref) on a B200.  This pins the
oracle: every reference entry point agrees to round-off.
"""
import numpy as np
import pytest

from oracle import ns3d_oracle as O

TOL = 1e-13  # relative L2; observed ~1e-16


def _grid(d):
    return O.Grid(int(d["Nx"]), int(d["Ny"]), int(d["Nz"]), float(d["Lx"]), float(d["Ly"]),
                  float(d["Lz"]))


CASES = ["iso16", "aniso16x8x24"]


@pytest.mark.parametrize("case", CASES)
def test_c2r_convention_matches_cufft(golden, case):
    d = golden[case]
    g = _grid(d)
    ours = O.c2r(g, d["X_nonherm"])
    ref = d["c2r_nonherm"]
    assert np.linalg.norm(ours - ref) / np.linalg.norm(ref) < TOL


@pytest.mark.parametrize("case", CASES)
def test_oracle_entry_points(golden, case):
    d = golden[case]
    g = _grid(d)
    Re, dt = float(d["Re"]), float(d["dt"])
    Uo, Vo, Ug, F = (list(d[k]) for k in ("U_odd", "V_odd", "U_gen", "F"))
    checks = {
        "conv_odd": O.convolution(g, Uo),
        "conv_gen": O.convolution(g, Ug),
        "conv_uv": O.convolution_uv(g, Uo, Vo),
        "rhs_odd": O.return_rhs(g, Uo, F, Re),
        "euler_odd": O.single_time_step(g, Uo, F, dt, Re),
        "rk3x1_odd": O.rk3_ssp(g, Uo, F, dt, Re),
        "rk3x1_gen": O.rk3_ssp(g, Ug, F, dt, Re),
        "linrhs_v": O.rk3_ssp_uv_rhs(g, Uo, Vo, dt, Re),
        "iuv_v": O.single_time_step_iuv_rhs(g, Uo, Vo, dt, Re),
    }
    U = Uo
    for _ in range(5):
        U = O.rk3_ssp(g, U, F, dt, Re)
    checks["rk3x5_odd"] = U
    un, vn = O.rk3_ssp_uv(g, Uo, Vo, F, dt, Re)
    checks["jvp_u"] = un
    checks["jvp_v"] = vn
    for k, mine in checks.items():
        err = O.rel_l2(mine, list(d[k]))
        assert err < TOL, (k, err)


@pytest.mark.parametrize("case", CASES)
def test_oracle_diagnostics(golden, case):
    d = golden[case]
    g = _grid(d)
    U = list(d["U_odd"])
    e, di = O.kinetic_energy(g, U), O.dissipation(g, U)
    assert abs(e / d["diag_odd"][0] - 1) < 1e-13
    assert abs(di / d["diag_odd"][1] - 1) < 1e-13


def test_krylov_pack_roundtrip(golden):
    d = golden["iso16"]
    g = _grid(d)
    V = list(d["V_odd"])
    vec = O.pack_reduced(V)
    assert vec.size == 3 * (g.Nx * g.Ny * g.Mz - 1)
    back = O.unpack_reduced(g, vec)
    # V is pure imaginary with V(0) = 0, so the round trip is exact
    for a, b in zip(back, V):
        assert np.array_equal(a, b)
