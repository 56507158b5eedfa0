"""CUDA path (through the C ABI) against the reference's golden vectors and the
oracle.  Tolerance: relative L2 <= 1e-12 for FP64 (the bar the reference
comparison sets); observed errors are ~1e-15.
"""
import math

import numpy as np
import pytest

from oracle import ns3d_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def torch():
    import torch as t

    if not t.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return t


def _np(F):
    return [f.detach().cpu().numpy() for f in F]


def _solver(g):
    from ns3dperiodic_b200 import Solver

    return Solver(g.Nx, g.Ny, g.Nz, g.Lx, g.Ly, g.Lz)


def _grid(d):
    return O.Grid(int(d["Nx"]), int(d["Ny"]), int(d["Nz"]), float(d["Lx"]), float(d["Ly"]),
                  float(d["Lz"]))


def _odd(g, seed, kmax=None):
    kmax = kmax if kmax is not None else min(g.Nx, g.Ny, g.Nz) / 3.0
    P = O.random_perturbation(g, seed, kmin=1.0, kmax=kmax)
    u = O.physical_velocity(g, P)
    s = 1.0 / math.sqrt(sum(float(np.mean(a * a)) for a in u) / 3.0)
    return [s * p for p in P]


def _general(g, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    jm = (-np.arange(g.Nx)) % g.Nx
    km = (-np.arange(g.Ny)) % g.Ny
    U = []
    for _ in range(3):
        w = rng.standard_normal(g.shape_c) + 1j * rng.standard_normal(g.shape_c)
        w *= g.mask  # fully populated inside the 2/3 sphere
        for l in (0, g.Nz // 2):
            P = w[:, :, l]
            w[:, :, l] = 0.5 * (P + np.conj(P[jm][:, km]))
        w[0, 0, 0] = 0
        U.append(w)
    U = O.leray_project(g, U)
    u = O.physical_velocity(g, U)
    s = 1.0 / math.sqrt(sum(float(np.mean(a * a)) for a in u) / 3.0)
    return [s * x for x in U]


# ---------------------------------------------------------------------------
# against the reference's own CUDA build (golden vectors)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("case", ["iso16", "aniso16x8x24"])
def test_entry_points_match_reference_golden(torch, golden, case):
    d = golden[case]
    g = _grid(d)
    Re, dt = float(d["Re"]), float(d["dt"])
    S = _solver(g)
    F = S.to_device(list(d["F"]))
    S.set_forcing(F)
    assert S.forcing_modes == 2

    def dev(k):
        return S.to_device(list(d[k]))

    def check(name, got):
        err = O.rel_l2(_np(got), list(d[name]))
        assert err < TOL, (name, err)

    check("conv_odd", S.calculate_convolution_2p3(dev("U_odd")))
    check("conv_gen", S.calculate_convolution_2p3(dev("U_gen")))
    check("conv_uv", S.calculate_convolution_2p3_uv(dev("U_odd"), dev("V_odd")))
    check("rhs_odd", S.return_rhs(dev("U_odd"), Re))
    check("euler_odd", S.single_time_step(dev("U_odd"), dt, Re))
    check("rk3x1_odd", S.rk3_ssp(dev("U_odd"), dt, Re))
    check("rk3x5_odd", S.rk3_ssp(dev("U_odd"), dt, Re, nsteps=5))
    check("rk3x1_gen", S.rk3_ssp(dev("U_gen"), dt, Re))
    U, V = S.rk3_ssp_uv(dev("U_odd"), dev("V_odd"), dt, Re)
    check("jvp_u", U)
    check("jvp_v", V)
    check("linrhs_v", S.rk3_ssp_uv_rhs(dev("U_odd"), dev("V_odd"), Re))
    check("iuv_v", S.single_time_step_iuv_rhs(dev("U_odd"), dev("V_odd"), dt, Re))
    e, di, _ = S.diagnostics(dev("U_odd"))
    assert abs(e / d["diag_odd"][0] - 1) < 1e-12
    assert abs(di / d["diag_odd"][1] - 1) < 1e-12
    S.close()


# ---------------------------------------------------------------------------
# every compiled extent against the oracle
# ---------------------------------------------------------------------------
GRIDS = [
    (8, 8, 8), (16, 16, 16), (24, 24, 24), (32, 32, 32), (48, 48, 48), (64, 64, 64),
    (96, 96, 96), (128, 128, 128), (32, 64, 48), (96, 16, 32), (8, 24, 16), (192, 16, 16),
    (16, 192, 24), (16, 16, 192), (256, 16, 16), (16, 256, 16), (16, 16, 256),
    (384, 8, 8), (8, 384, 8), (8, 8, 384), (512, 8, 8), (8, 512, 8), (8, 8, 512),
]


@pytest.mark.parametrize("shape", GRIDS, ids=lambda s: "x".join(map(str, s)))
def test_rk3_and_convolution_vs_oracle(torch, shape):
    Nx, Ny, Nz = shape
    g = O.Grid(Nx, Ny, Nz, 2 * math.pi, 4.0, 3.0)
    U = _general(g, 7)
    F = O.kolmogorov_forcing(g, 2)
    Re, dt = 120.0, 2e-3
    S = _solver(g)
    S.set_forcing(S.to_device(F))
    Q = _np(S.calculate_convolution_2p3(S.to_device(U)))
    assert O.rel_l2(Q, O.convolution(g, U)) < TOL
    Ud = S.rk3_ssp(S.to_device(U), dt, Re)
    assert O.rel_l2(_np(Ud), O.rk3_ssp(g, U, F, dt, Re)) < TOL
    S.close()


@pytest.mark.parametrize("shape", [(16, 16, 16), (24, 32, 16), (48, 48, 48), (64, 64, 64),
                                   (96, 32, 64), (8, 8, 384), (8, 8, 512)],
                         ids=lambda s: "x".join(map(str, s)))
def test_tangent_steppers_vs_oracle(torch, shape):
    Nx, Ny, Nz = shape
    g = O.Grid(Nx, Ny, Nz)
    U = _odd(g, 3)
    V = _odd(g, 4)
    F = O.kolmogorov_forcing(g, 2)
    Re, dt = 90.0, 3e-3
    S = _solver(g)
    S.set_forcing(S.to_device(F))
    Q = _np(S.calculate_convolution_2p3_uv(S.to_device(U), S.to_device(V)))
    assert O.rel_l2(Q, O.convolution_uv(g, U, V)) < TOL
    Un, Vn = S.rk3_ssp_uv(S.to_device(U), S.to_device(V), dt, Re)
    ou, ov = O.rk3_ssp_uv(g, U, V, F, dt, Re)
    assert O.rel_l2(_np(Un), ou) < TOL
    assert O.rel_l2(_np(Vn), ov) < TOL
    Vl = S.rk3_ssp_uv_rhs(S.to_device(U), S.to_device(V), Re)
    assert O.rel_l2(_np(Vl), O.rk3_ssp_uv_rhs(g, U, V, dt, Re)) < TOL
    Vi = S.single_time_step_iuv_rhs(S.to_device(U), S.to_device(V), dt, Re)
    assert O.rel_l2(_np(Vi), O.single_time_step_iuv_rhs(g, U, V, dt, Re)) < TOL
    S.close()


# ---------------------------------------------------------------------------
# analytic and structural checks
# ---------------------------------------------------------------------------
def test_shapiro_32_100_steps(torch):
    """Shapiro's exact Beltrami solution: rel L2 < 1e-10, divergence at round-off."""
    g = O.Grid(32, 32, 32)
    Re, dt = 100.0, 1e-3
    S = _solver(g)
    U = S.rk3_ssp(S.to_device(O.shapiro_hat(g, 0.0, Re)), dt, Re, nsteps=100)
    err = O.rel_l2(_np(U), O.shapiro_hat(g, 100 * dt, Re))
    assert err < 1e-10, err
    _, _, div = S.diagnostics(U)
    umax = max(float(u.abs().max()) for u in U)
    assert div < 1e-13 * umax


def test_graph_replay_equals_single_steps(torch):
    g = O.Grid(32, 32, 32)
    U = _general(g, 11)
    S = _solver(g)
    S.set_forcing(S.to_device(O.kolmogorov_forcing(g, 4)))
    A = S.rk3_ssp(S.to_device(U), 1e-3, 200.0, nsteps=4)
    B = S.to_device(U)
    for _ in range(4):
        S.rk3_ssp(B, 1e-3, 200.0)
    for a, b in zip(A, B):
        assert torch.equal(a, b)


def test_krylov_adapters_vs_oracle(torch):
    g = O.Grid(16, 16, 16)
    U = _odd(g, 5)
    V = _odd(g, 6)
    Re, tau = 75.0, 0.5
    S = _solver(g)
    vec = torch.as_tensor(O.pack_reduced(V)).to("cuda")
    Vd = S.unpack_reduced(vec)
    assert O.rel_l2(_np(Vd), V) == 0.0
    assert torch.equal(S.pack_reduced(Vd), vec)
    out = S.matvec_reduced(S.to_device(U), vec, Re)
    ref = O.linearised_matvec_reduced(g, U, O.pack_reduced(V), 0.0, Re)
    assert np.linalg.norm(out.cpu().numpy() - ref) / np.linalg.norm(ref) < TOL
    out2 = S.matvec_reduced(S.to_device(U), vec, Re, tau=tau)
    ref2 = ref - O.pack_reduced(V) / tau  # A_vector_add_diagonal_kernel
    assert np.linalg.norm(out2.cpu().numpy() - ref2) / np.linalg.norm(ref2) < TOL


def test_diagnostics_vs_oracle(torch):
    g = O.Grid(32, 48, 24, 3.0, 2 * math.pi, 5.0)
    U = _general(g, 9)
    S = _solver(g)
    e, d, dv = S.diagnostics(S.to_device(U))
    assert abs(e / O.kinetic_energy(g, U) - 1) < 1e-12
    assert abs(d / O.dissipation(g, U) - 1) < 1e-12
    ref_div = float(np.abs(O.divergence_hat(g, U)).max())
    assert abs(dv - ref_div) <= 1e-12 * max(1.0, ref_div) + 1e-9


def test_dense_forcing_path(torch):
    """Forcing with more non-zero modes than the sparse list holds."""
    g = O.Grid(32, 32, 32)
    rng = np.random.Generator(np.random.PCG64(1))
    F = [1j * rng.standard_normal(g.shape_c) for _ in range(3)]
    U = _general(g, 2)
    S = _solver(g)
    Fd = S.to_device(F)
    S.set_forcing(Fd)
    assert S.forcing_modes == -1
    Ud = S.rk3_ssp(S.to_device(U), 1e-3, 100.0)
    assert O.rel_l2(_np(Ud), O.rk3_ssp(g, U, F, 1e-3, 100.0)) < TOL
    R = S.return_rhs(S.to_device(U), 100.0)
    assert O.rel_l2(_np(R), O.return_rhs(g, U, F, 100.0)) < TOL


def test_errors_are_status_codes(torch):
    from ns3dperiodic_b200 import Ns3dError, Solver

    with pytest.raises(Ns3dError) as e:
        Solver(100, 64, 64)
    assert e.value.status == 2
    S = Solver(16, 16, 16)
    U = S.zeros()
    with pytest.raises(Ns3dError) as e:
        S.rk3_ssp(U, 1e-3, -1.0)
    assert e.value.status == 1
    with pytest.raises(ValueError):
        S.rk3_ssp([u.cpu() for u in U], 1e-3, 1.0)
    S.close()
