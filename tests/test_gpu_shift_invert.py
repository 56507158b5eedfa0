"""Shift-invert maps and the matrix-exponent implicit restart on the GPU
(through the C ABI) against the oracle and the reference's own
Implicit_restart_Arnoldi_GPU_data_Matrix_Exponent
(tests/golden/krylov_shift_invert.npz).

Tolerances: the forward maps are linear in the tangent step, so they match
the oracle to round-off (rel L2 < 1e-12).  The inverse maps are BiCGStab(L)
solves to a relative residual of 1e-9 (the reference's BiCG_tol), checked
through the oracle's forward map (< 5e-9).  Converged eigenvalues agree with
the reference's to 1e-8 (IRA tolerance 5e-8 on Ritz estimates, a
well-conditioned spectrum).
"""
import math
import os

import numpy as np
import pytest

from oracle import krylov_oracle as K
from oracle import ns3d_oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SIGMA, THETA = 1.05, 0.05


@pytest.fixture(scope="module")
def torch():
    import torch as t

    if not t.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return t


@pytest.fixture(scope="module")
def ns16():
    """16^3 Kolmogorov base flow at Re = 40, the solver and device copies.
    dt = 1e-3 keeps sigma = 1.05 outside the spectrum of E (3 implicit steps
    move it by about 3 dt |J| ~ 0.06 from 1), where the inner solves converge
    in a few iterations; at dt = 0.02 they diverge, on the oracle too."""
    from ns3dperiodic_b200 import Solver

    g = O.Grid(16, 16, 16)
    Re, dt, steps = 40.0, 1.0e-3, 3
    U, _ = O.kolmogorov_state(g, Re, 5, rel_amp=1e-2)
    S = Solver(16, 16, 16)
    Ud = S.to_device(U)
    Vs = S.zeros()
    yield g, U, S, Ud, Vs, Re, dt, steps
    S.close()


def _kr(n, m):
    from ns3dperiodic_b200.krylov import Krylov

    return Krylov(n, m)


@pytest.mark.parametrize("rotated", [False, True])
def test_shifted_maps_match_oracle(torch, ns16, rotated):
    g, U, S, Ud, Vs, Re, dt, steps = ns16
    n = S.krylov_length
    nn = 2 * n if rotated else n
    kr = _kr(nn, 2)
    A = kr.exponential_shifted_map(S, Ud, Vs, dt, Re, steps, SIGMA,
                                   THETA if rotated else None)
    x = np.random.default_rng(21).standard_normal(nn)
    y = torch.empty(nn, dtype=torch.float64, device="cuda")
    kr.apply(A, torch.as_tensor(x, device="cuda"), y)
    assert A.status == 0
    if rotated:
        want = O.exponential_rotated_reduced(g, U, x, dt, Re, steps, SIGMA, THETA)
    else:
        want = O.exponential_shifted_reduced(g, U, x, dt, Re, steps, SIGMA)
    assert O.rel_l2(y.cpu().numpy(), want) < 1e-12
    # the base flow stays fixed
    assert O.rel_l2([u.cpu().numpy() for u in Ud], U) == 0.0
    kr.close()


def test_rotated_map_is_the_complex_shift(torch, ns16):
    """The rotated map is the real form of (E - sigma e^{i theta}) acting on
    x_r + i x_i: its halves follow from the unrotated map with shift 0."""
    g, U, S, Ud, Vs, Re, dt, steps = ns16
    n = S.krylov_length
    rng = np.random.default_rng(22)
    xr, xi = rng.standard_normal(n), rng.standard_normal(n)
    kr1, kr2 = _kr(n, 2), _kr(2 * n, 2)
    E = kr1.exponential_shifted_map(S, Ud, Vs, dt, Re, steps, 0.0)
    Rm = kr2.exponential_shifted_map(S, Ud, Vs, dt, Re, steps, SIGMA, THETA)
    er = torch.empty(n, dtype=torch.float64, device="cuda")
    ei = torch.empty_like(er)
    kr1.apply(E, torch.as_tensor(xr, device="cuda"), er)
    kr1.apply(E, torch.as_tensor(xi, device="cuda"), ei)
    out = torch.empty(2 * n, dtype=torch.float64, device="cuda")
    kr2.apply(Rm, torch.as_tensor(np.concatenate([xr, xi]), device="cuda"), out)
    s = SIGMA * complex(math.cos(THETA), math.sin(THETA))
    z = (er.cpu().numpy() + 1j * ei.cpu().numpy()) - s * (xr + 1j * xi)
    o = out.cpu().numpy()
    assert O.rel_l2(o[:n], z.real) < 1e-13
    assert O.rel_l2(o[n:], z.imag) < 1e-13
    kr1.close()
    kr2.close()


@pytest.mark.parametrize("rotated", [False, True])
def test_exponent_invert_solves_the_shifted_system(torch, ns16, rotated):
    g, U, S, Ud, Vs, Re, dt, steps = ns16
    n = S.krylov_length
    nn = 2 * n if rotated else n
    kr = _kr(nn, 2)
    angle = THETA if rotated else None
    Ainv = kr.exponent_invert_map(S, Ud, Vs, dt, Re, steps, SIGMA, angle, L=6, tol=1e-9)
    b = np.random.default_rng(23).standard_normal(nn)
    x = torch.full((nn,), float("nan"), dtype=torch.float64, device="cuda")
    kr.apply(Ainv, torch.as_tensor(b, device="cuda"), x)
    st = Ainv.stats()
    assert Ainv.status == 0 and st["last_flag"] == 0 and st["solves"] == 1
    assert st["last_tol"] < 1e-9
    xs = x.cpu().numpy()
    if rotated:
        Ax = O.exponential_rotated_reduced(g, U, xs, dt, Re, steps, SIGMA, THETA)
    else:
        Ax = O.exponential_shifted_reduced(g, U, xs, dt, Re, steps, SIGMA)
    assert np.linalg.norm(Ax - b) / np.linalg.norm(b) < 5e-9
    # warm start from the solution: the solve stops before its first iteration
    W = kr.exponent_invert_map(S, Ud, Vs, dt, Re, steps, SIGMA, angle, tol=1e-6,
                               warm_start=True)
    x2 = x.clone()
    kr.apply(W, torch.as_tensor(b, device="cuda"), x2)
    assert W.status == 0 and W.stats()["last_iter"] == 0
    assert torch.equal(x2, x)
    kr.close()


def test_exponent_invert_reports_no_convergence(torch, ns16):
    """The reference exits when its inner solve fails; the map records
    status 7 and fills its output with NaN, so the driver stops."""
    from ns3dperiodic_b200._lib import Ns3dError

    g, U, S, Ud, Vs, Re, dt, steps = ns16
    n = S.krylov_length
    kr = _kr(n, 6)
    Ainv = kr.exponent_invert_map(S, Ud, Vs, dt, Re, steps, SIGMA, L=1, tol=1e-15, max_iter=1)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    b = torch.as_tensor(np.random.default_rng(24).standard_normal(n), device="cuda")
    kr.apply(Ainv, b, x)
    assert Ainv.status == 7 and Ainv.stats()["last_flag"] == 1
    assert torch.isnan(x).all()
    A = kr.linearised_map(S, Ud, Re)
    with pytest.raises(Ns3dError):
        kr.implicit_restart_arnoldi_matrix_exponent(Ainv, A, k=2, m=6, max_iter=2)
    kr.close()


def _golden():
    return np.load(os.path.join(GOLDEN, "krylov_shift_invert.npz"))


def _set_distance(a, b) -> float:
    """Largest distance when each value of a is matched to the nearest still
    unmatched value of b (eigenvalues as multisets; conjugate pairs with equal
    real parts make sorting unreliable)."""
    b = list(np.asarray(b))
    worst = 0.0
    for x in np.asarray(a):
        j = int(np.argmin([abs(x - y) for y in b]))
        worst = max(worst, abs(x - b.pop(j)))
    return worst


def _rayleigh(A, X):
    lam = np.array([np.vdot(x, A @ x) / np.vdot(x, x) for x in X])
    res = np.array([np.linalg.norm(A @ x - l * x) / np.linalg.norm(x) for x, l in zip(X, lam)])
    return lam, res


@pytest.mark.parametrize("tag", ["plain", "rotated"])
def test_matrix_exponent_ira_matches_reference_golden(torch, tag):
    """The whole driver with dense operators against the reference's
    Implicit_restart_Arnoldi_GPU_data_Matrix_Exponent: the same converged
    eigenvalues of the original map (the reference's from Rayleigh quotients
    of its eigenvectors), and eigenvectors with small residuals."""
    z = _golden()
    A, Minv = z["A"], z[f"Minv_{tag}"]
    k, m, tol = int(z["k"]), int(z["m"]), float(z["tol"])
    n = A.shape[0]
    rotated = tag == "rotated"
    kr = _kr(Minv.shape[0], m)
    half = _kr(n, 2)
    Md, Ad = torch.as_tensor(Minv, device="cuda"), torch.as_tensor(A, device="cuda")
    Mmap = kr.python_map(lambda x, y: torch.mv(Md, x, out=y))
    Amap = half.python_map(lambda x, y: torch.mv(Ad, x, out=y))
    out = kr.implicit_restart_arnoldi_matrix_exponent(Mmap, Amap, "LR", "LM", k, m, tol, 200,
                                                      rotated=rotated, seed=3)
    assert out["ritz_norm"] <= tol
    lam_ref, res_ref = _rayleigh(A, z[f"vec_re_{tag}"] + 1j * z[f"vec_im_{tag}"])
    assert res_ref.max() < 1e-8
    w = out["eigenvalues"]
    assert _set_distance(w, lam_ref) < 1e-8
    X = out["eigenvectors"].cpu().numpy()
    for i in range(k):
        assert np.linalg.norm(A @ X[i] - w[i] * X[i]) < 1e-8 * np.linalg.norm(X[i])
    # the residuals the final stage reports are the reference's Schur residuals
    assert out["residual_real"].max() < 1e-8 and out["residual_imag"].max() < 1e-8
    # and the same driver on the oracle gives the same eigenvalues
    o = K.ira_matrix_exponent(lambda v: Minv @ v, lambda v: A @ v, Minv.shape[0], k, m, "LR",
                              "LM", tol, 200, rotated=rotated, seed=3)
    assert _set_distance(o["eigenvalues"], w) < 1e-8
    kr.close()
    half.close()


def test_rotated_final_stage_on_the_ns_operator_matches_oracle(torch, ns16):
    """A short rotated shift-invert restart on the 16^3 Navier-Stokes maps,
    then the final stage on the linearised map: the GPU path and the oracle's
    restatement of compute_eigensystem_of_original_mapping_rotation agree on
    the same Krylov basis."""
    g, U, S, Ud, Vs, Re, dt, steps = ns16
    n = S.krylov_length
    k, m = 2, 6
    kr = _kr(2 * n, m)
    Ainv = kr.exponent_invert_map(S, Ud, Vs, dt, Re, steps, SIGMA, THETA, tol=1e-9)
    A = kr.linearised_map(S, Ud, Re)
    eig, rn, it, V, H = kr.implicit_restart_arnoldi(Ainv, "LM", k=k, m=m, tol=1e-12,
                                                    max_iter=2, seed=4)
    assert Ainv.status == 0 and Ainv.stats()["solves"] > 0
    w, X, rr, ri = kr.eigenpairs_rotated(A, V, H, k, "LR")
    V1 = K.schur_basis(V.cpu().numpy(), H, k)
    wo, Xo, rro, rio = K.eigensystem_rotation(
        lambda v: O.linearised_matvec_reduced(g, U, v, 0.0, Re), V1, "LR")
    scale = max(np.abs(wo).max(), 1.0)
    assert _set_distance(w, wo) < 1e-10 * scale
    assert np.abs(rr - rro).max() < 1e-9 * max(rro.max(), 1.0)
    assert np.abs(ri - rio).max() < 1e-9 * max(rio.max(), 1.0)
    kr.close()
