"""Krylov path on the GPU (through the C ABI) against the reference's own
Arnoldi_driver outputs (tests/golden/krylov_arnoldi.npz) and the oracle.

Tolerances: H within 1e-12 of its largest entry, V and f within 1e-11
absolute (unit-norm columns) for the golden cases; the GPU dot products sum
in a different order than cuBLAS, so agreement is at round-off (~1e-15),
growing slowly with the column index.
"""
import math
import os

import numpy as np
import pytest

from oracle import krylov_oracle as K
from oracle import ns3d_oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def torch():
    import torch as t

    if not t.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return t


def _kr(n, m):
    from ns3dperiodic_b200.krylov import Krylov

    return Krylov(n, m)


def _dense(n, seed):
    return np.random.default_rng(seed).standard_normal((n, n)) / np.sqrt(n)


def _torch_dense_map(torch, kr, A):
    Ad = torch.as_tensor(A, device="cuda")
    return kr.python_map(lambda x, y: torch.mv(Ad, x, out=y))


@pytest.mark.parametrize("name", ["laplace", "dense"])
def test_arnoldi_matches_reference_golden(torch, name):
    """From k = 0, then continued from k = kc with a random residual that is
    not orthogonal to the kept columns.  For the dense matrix that drives
    every later column to the 13-pass reorthogonalisation limit (the
    reference prints "Arnoldi orthogonalization failed" there and goes on)."""
    d = np.load(os.path.join(GOLDEN, "krylov_arnoldi.npz"))
    n, m, kc, seed = (int(x) for x in d[f"{name}_meta"])
    kr = _kr(n, m)
    A = kr.laplace_map() if name == "laplace" else _torch_dense_map(torch, kr, _dense(n, seed))
    V = torch.zeros((m, n), dtype=torch.float64, device="cuda")
    H = np.zeros((m, m))
    f = torch.as_tensor(d[f"{name}_f0"], device="cuda").clone()
    st = kr.arnoldi(A, V, H, f, 0, m)
    assert st["limit_hits"] == 0
    sc = np.abs(d[f"{name}_H"]).max()
    assert np.abs(H - d[f"{name}_H"]).max() < 1e-12 * sc
    assert np.abs(V.cpu().numpy() - d[f"{name}_V"]).max() < 1e-11
    assert np.abs(f.cpu().numpy() - d[f"{name}_f"]).max() < 1e-11 * max(
        1.0, np.abs(d[f"{name}_f"]).max())
    V = torch.as_tensor(d[f"{name}_cont_V_in"], device="cuda").clone()
    H = d[f"{name}_cont_H_in"].copy()
    f = torch.as_tensor(d[f"{name}_cont_f_in"], device="cuda").clone()
    st = kr.arnoldi(A, V, H, f, kc, m)
    if name == "dense":
        assert st["limit_hits"] == m - kc - 1 and st["max_passes"] == 13
    assert np.abs(H - d[f"{name}_cont_H"]).max() < 1e-12 * sc
    assert np.abs(V.cpu().numpy() - d[f"{name}_cont_V"]).max() < 1e-11
    kr.close()


def test_laplace_map_matches_reference_golden(torch):
    d = np.load(os.path.join(GOLDEN, "krylov_arnoldi.npz"))
    x = d["laplace_apply_in"]
    kr = _kr(x.size, 2)
    A = kr.laplace_map()
    # apply through a 2-column Arnoldi: w = A v with v = x/||x||, H(0,0) = v.Av
    V = torch.zeros((2, x.size), dtype=torch.float64, device="cuda")
    H = np.zeros((2, 2))
    f = torch.as_tensor(x, device="cuda").clone()
    kr.arnoldi(A, V, H, f, 0, 2)
    v = x / np.linalg.norm(x)
    ref = d["laplace_apply_out"] / np.linalg.norm(x)
    assert abs(H[0, 0] - v @ ref) < 1e-13
    kr.close()


@pytest.mark.parametrize("n,m", [(1 << 20, 20), ((1 << 18) + 7, 33)])
def test_arnoldi_large_vs_oracle(torch, n, m):
    """Vectors larger than L2 (8 MB each, ragged length) and more than 32 columns."""
    kr = _kr(n, m)
    rng = np.random.default_rng(n)
    f0 = rng.standard_normal(n)
    V = torch.zeros((m, n), dtype=torch.float64, device="cuda")
    H = np.zeros((m, m))
    f = torch.as_tensor(f0, device="cuda").clone()
    kr.arnoldi(kr.laplace_map(), V, H, f, 0, m)
    Vo, Ho, fo = np.zeros((m, n)), np.zeros((m, m)), f0.copy()
    K.arnoldi_driver(K.laplace1d, Vo, Ho, fo, 0, m)
    assert np.abs(H - Ho).max() < 1e-11 * np.abs(Ho).max()
    assert np.abs(V.cpu().numpy() - Vo).max() < 1e-10
    Vg = V.cpu().numpy()
    assert np.abs(Vg @ Vg.T - np.eye(m)).max() < 1e-13
    kr.close()


def _kolmogorov(g, Re, seed):
    U, _ = O.kolmogorov_state(g, Re, seed, rel_amp=1e-2)
    return U


def test_arnoldi_linearised_ns_vs_oracle(torch):
    from ns3dperiodic_b200 import Solver

    g = O.Grid(16, 16, 16)
    Re = 40.0
    U = _kolmogorov(g, Re, 3)
    S = Solver(16, 16, 16)
    Ud = S.to_device(U)
    n = S.krylov_length
    m = 10
    kr = _kr(n, m)
    A = kr.linearised_map(S, Ud, Re)
    f0 = np.random.default_rng(4).standard_normal(n)
    V = torch.zeros((m, n), dtype=torch.float64, device="cuda")
    H = np.zeros((m, m))
    f = torch.as_tensor(f0, device="cuda").clone()
    kr.arnoldi(A, V, H, f, 0, m)
    assert A.status == 0
    Vo, Ho, fo = np.zeros((m, n)), np.zeros((m, m)), f0.copy()
    K.arnoldi_driver(lambda v: O.linearised_matvec_reduced(g, U, v, 0.0, Re), Vo, Ho, fo, 0, m)
    assert np.abs(H - Ho).max() < 1e-10 * np.abs(Ho).max()
    assert np.abs(V.cpu().numpy() - Vo).max() < 1e-9
    kr.close()
    S.close()


def test_arnoldi_exponential_map_vs_oracle(torch):
    """Tangent map over `steps` Heun steps; the base flow advances per call."""
    from ns3dperiodic_b200 import Solver

    g = O.Grid(16, 16, 16)
    Re, dt, steps, m = 40.0, 5e-3, 2, 5
    U = _kolmogorov(g, Re, 7)
    F = O.kolmogorov_forcing(g)
    S = Solver(16, 16, 16)
    S.set_forcing(S.to_device(F))
    Ud = S.to_device(U)
    Vs = S.zeros()
    n = S.krylov_length
    kr = _kr(n, m)
    A = kr.exponential_map(S, Ud, Vs, dt, Re, steps)
    f0 = np.random.default_rng(8).standard_normal(n)
    V = torch.zeros((m, n), dtype=torch.float64, device="cuda")
    H = np.zeros((m, m))
    f = torch.as_tensor(f0, device="cuda").clone()
    kr.arnoldi(A, V, H, f, 0, m)
    assert A.status == 0
    state = {"U": U}

    def oracle_map(v):
        W = O.unpack_reduced(g, v)
        Ub = state["U"]
        for _ in range(steps):
            Ub, W = O.rk3_ssp_uv(g, Ub, W, F, dt, Re)
        state["U"] = Ub
        return O.pack_reduced(W)

    Vo, Ho, fo = np.zeros((m, n)), np.zeros((m, m)), f0.copy()
    K.arnoldi_driver(oracle_map, Vo, Ho, fo, 0, m)
    assert np.abs(H - Ho).max() < 1e-10 * np.abs(Ho).max()
    assert O.rel_l2([u.cpu().numpy() for u in Ud], state["U"]) < 1e-12
    kr.close()
    S.close()


def test_restart_matches_oracle(torch):
    from ns3dperiodic_b200 import krylov as KR

    n, m, k = 5000, 16, 5
    rng = np.random.default_rng(12)
    X = np.eye(400) + 0.1 * rng.standard_normal((400, 400))
    A400 = X @ np.diag(np.linspace(1.0, 0.05, 400)) @ np.linalg.inv(X)
    # a factorisation of a block operator of size n (A400 on the first 400 rows)
    Vo, Ho, fo = np.zeros((m, n)), np.zeros((m, m)), rng.standard_normal(n)

    def Ax(v):
        w = 0.5 * v.copy()
        w[:400] = A400 @ v[:400]
        return w

    K.arnoldi_driver(Ax, Vo, Ho, fo, 0, m)
    eig, _ = KR.select_shifts(Ho, "LR")
    Q, Hn, k0 = KR.qr_shifts(k, Ho, eig)
    kr = _kr(n, m)
    V = torch.as_tensor(Vo, device="cuda").clone()
    f = torch.as_tensor(fo, device="cuda").clone()
    Qg = Q.copy()
    fn = kr.ira_restart(V, f, Qg, Hn, k0)
    Qo = Q.copy()
    fno = K.ira_restart(Vo, fo, Qo, Hn, k0)
    assert abs(fn / fno - 1.0) < 1e-13
    np.testing.assert_array_equal(Qg, Qo)
    assert np.abs(V.cpu().numpy() - Vo).max() < 1e-13
    assert np.abs(f.cpu().numpy() - fo).max() < 1e-13 * max(1.0, np.abs(fo).max())
    kr.close()


def test_implicit_restart_finds_leading_eigenvalues(torch):
    """IRA loop (host mirror) on a non-normal operator with known spectrum."""
    n = 400
    rng = np.random.default_rng(13)
    lam = np.concatenate([[2.0, 1.8, 1.7 + 0.3j, 1.7 - 0.3j], np.linspace(1.0, 0.01, n - 4)])
    D = np.diag(lam.real)
    D[2, 3], D[3, 2] = 0.3, -0.3
    X = np.eye(n) + 0.05 * rng.standard_normal((n, n))
    A = X @ D @ np.linalg.inv(X)
    kr = _kr(n, 20)
    eig, rn, it, V, H = kr.implicit_restart_arnoldi(_torch_dense_map(torch, kr, A), "LR", k=4,
                                                    m=20, tol=1e-10, max_iter=200, seed=1)
    assert rn <= 1e-10
    got = np.sort_complex(eig[:4])
    want = np.sort_complex(np.array([2.0, 1.8, 1.7 + 0.3j, 1.7 - 0.3j]))
    assert np.abs(got - want).max() < 1e-8
    kr.close()


def test_krylov_errors_are_status_codes(torch):
    from ns3dperiodic_b200 import Ns3dError

    n, m = 1000, 6
    kr = _kr(n, m)
    V = torch.zeros((m, n), dtype=torch.float64, device="cuda")
    H = np.zeros((m, m))
    f = torch.zeros(n, dtype=torch.float64, device="cuda")
    with pytest.raises(Ns3dError) as e:  # ||f|| < 1e-15 at k = 0
        kr.arnoldi(kr.laplace_map(), V, H, f, 0, m)
    assert e.value.status == 1
    f.normal_()
    with pytest.raises(Ns3dError) as e:  # k >= m
        kr.arnoldi(kr.laplace_map(), V, H, f, m, m)
    assert e.value.status == 1
    nan_map = kr.python_map(lambda x, y: y.fill_(math.nan))
    with pytest.raises(Ns3dError) as e:
        kr.arnoldi(nan_map, V, H, f, 0, m)
    assert e.value.status == 5
    with pytest.raises(ValueError):
        kr.arnoldi(kr.laplace_map(), V.cpu(), H, f, 0, m)
    kr.close()


@pytest.mark.parametrize("k0", [1, 7, 8, 9, 16, 17, 33, 64, 70])
def test_restart_all_kernel_widths(torch, k0):
    """Every width of the register-tiled restart (k0 <= 8, 16, 32, 64) and the
    shared-memory form beyond, against the oracle's V Q and f update."""
    n, m = 3001, 80
    rng = np.random.default_rng(100 + k0)
    Vo = rng.standard_normal((m, n))
    fo = rng.standard_normal(n)
    Q = np.linalg.qr(rng.standard_normal((m, m)))[0]
    H = np.triu(rng.standard_normal((m, m)), -1)
    kr = _kr(n, m)
    V = torch.as_tensor(Vo, device="cuda").clone()
    f = torch.as_tensor(fo, device="cuda").clone()
    Qg = Q.copy()
    fn = kr.ira_restart(V, f, Qg, H, k0)
    Qo = Q.copy()
    fno = K.ira_restart(Vo, fo, Qo, H, k0)
    assert abs(fn / fno - 1.0) < 1e-13
    assert np.abs(V.cpu().numpy() - Vo).max() < 1e-12
    assert np.abs(f.cpu().numpy() - fo).max() < 1e-12
    kr.close()


def _lin_matrix(n, seed, diag, scale):
    rng = np.random.default_rng(seed)
    return diag * np.eye(n) + scale * rng.standard_normal((n, n)) / np.sqrt(n)


@pytest.mark.parametrize("idx", range(3))
def test_bicgstabl_matches_reference_golden(torch, idx):
    d = np.load(os.path.join(GOLDEN, "krylov_linsolve.npz"))
    n, L, seed, flag, it = (int(v) for v in d[f"bicg{idx}_meta"])
    kr = _kr(n, 4)
    A = _torch_dense_map(torch, kr, _lin_matrix(n, seed, 2.0, 0.5))
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    b = torch.as_tensor(d[f"bicg{idx}_b"], device="cuda")
    fl, its, err = kr.bicgstabl(A, x, b, L, 1e-10, 200)
    assert (fl, its) == (flag, it)
    ref = d[f"bicg{idx}_x"]
    assert np.abs(x.cpu().numpy() - ref).max() < 1e-10 * np.abs(ref).max()
    kr.close()


def test_newton_matches_reference_golden(torch):
    d = np.load(os.path.join(GOLDEN, "krylov_linsolve.npz"))
    n, seed, flag, it = (int(v) for v in d["newton_meta"])
    c, tol_out = (float(v) for v in d["newton_c_tol"])
    Ad = torch.as_tensor(_lin_matrix(n, seed, 3.0, 0.3), device="cuda")
    bd = torch.as_tensor(d["newton_b"], device="cuda")
    base = torch.zeros(n, dtype=torch.float64, device="cuda")
    kr = _kr(n, 4)

    def residual(x, y):
        base.copy_(x)
        torch.mv(Ad, x, out=y)
        y.add_(c * x ** 3 - bd)

    def jacobian(v, y):
        torch.mv(Ad, v, out=y)
        y.add_(3.0 * c * base ** 2 * v)

    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    r = kr.newton(kr.python_map(jacobian), kr.python_map(residual), x, 1e-9, 60, 1e-11, 200)
    assert (r["flag"], r["iterations"], r["linsolve_flag"]) == (flag, it, 0)
    assert abs(r["tol"] - tol_out) < 1e-6 * tol_out + 1e-14
    ref = d["newton_x"]
    assert np.abs(x.cpu().numpy() - ref).max() < 1e-10 * np.abs(ref).max()
    kr.close()


def test_newton_finds_the_laminar_kolmogorov_flow(torch):
    """F(u) = RHS(u) on reduced vectors (ns3d_map_rhs) with the linearised map
    on the same base flow as the Jacobian: from a perturbed start, Newton
    returns to the laminar fixed point u = (Re/16) sin(4y) x."""
    from ns3dperiodic_b200 import Solver

    g = O.Grid(16, 16, 16)
    Re = 5.0
    U0, F = O.kolmogorov_state(g, Re, 0, rel_amp=0.0)
    P = O.random_perturbation(g, 4)
    Ustart = [U0[i] + 0.05 * P[i] for i in range(3)]
    S = Solver(16, 16, 16)
    S.set_forcing(S.to_device(F))
    n = S.krylov_length
    kr = _kr(n, 4)
    Ub = S.zeros()
    Vs = S.zeros()
    Fm = kr.rhs_map(S, Ub, Vs, Re)
    Jm = kr.linearised_map(S, Ub, Re)
    x = torch.as_tensor(O.pack_reduced(Ustart), device="cuda").clone()
    r = kr.newton(Jm, Fm, x, 1e-10, 80, 1e-12, 300)
    assert r["flag"] == 0 and Fm.status == 0 and Jm.status == 0
    ref = O.pack_reduced(U0)
    assert np.abs(x.cpu().numpy() - ref).max() < 1e-8 * np.abs(ref).max()
    kr.close()
    S.close()


def test_bicgstabl_reports_nan_and_bad_arguments(torch):
    from ns3dperiodic_b200 import Ns3dError

    n = 500
    kr = _kr(n, 4)
    b = torch.ones(n, dtype=torch.float64, device="cuda")
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    nan_map = kr.python_map(lambda v, y: y.fill_(math.nan))
    fl, its, err = kr.bicgstabl(nan_map, x, b, 2, 1e-8, 10)
    assert fl == -3
    with pytest.raises(Ns3dError) as e:
        kr.bicgstabl(nan_map, x, b, 0, 1e-8, 10)
    assert e.value.status == 1
    kr.close()


def test_combine_matches_numpy(torch):
    n, m, p = 7001, 12, 9
    rng = np.random.default_rng(21)
    Vo = rng.standard_normal((m, n))
    C = rng.standard_normal((m, p))
    kr = _kr(n, m)
    W = kr.combine(torch.as_tensor(Vo, device="cuda"), C)
    assert np.abs(W.cpu().numpy() - C.T @ Vo).max() < 1e-12 * np.abs(C.T @ Vo).max()
    kr.close()


def test_eigenpairs_of_the_implicit_restart(torch):
    """IRA to convergence, then the Schur / Galerkin stage: eigenvalues and
    eigenvectors of a non-normal operator with a known spectrum (a complex
    pair included) against numpy's dense eigen-decomposition."""
    n = 400
    rng = np.random.default_rng(13)
    lam = np.concatenate([[2.0, 1.8, 1.7, 1.7], np.linspace(1.0, 0.01, n - 4)])
    D = np.diag(lam)
    D[2, 3], D[3, 2] = 0.3, -0.3
    X = np.eye(n) + 0.05 * rng.standard_normal((n, n))
    A = X @ D @ np.linalg.inv(X)
    kr = _kr(n, 20)
    Am = _torch_dense_map(torch, kr, A)
    eig, rn, it, V, H = kr.implicit_restart_arnoldi(Am, "LR", k=4, m=20, tol=1e-11,
                                                    max_iter=300, seed=1)
    w, Xv, res = kr.eigenpairs(Am, V, H, 4, "LR")
    want = np.array([2.0, 1.8, 1.7 + 0.3j, 1.7 - 0.3j])
    assert np.abs(np.sort_complex(w) - np.sort_complex(want)).max() < 1e-8
    assert res.max() < 1e-8
    Xn = Xv.cpu().numpy()
    for i in range(4):
        x = Xn[i]
        r = A @ x - w[i] * x
        assert np.linalg.norm(r) < 1e-8 * np.linalg.norm(x)
    kr.close()


def test_restart_after_a_smaller_workspace_is_created(torch):
    """Kernel shared-memory caps are per kernel, not per workspace: a
    workspace created later with a small m_max (the inner solves of the
    shift-invert maps use m_max = 2) must not break the restart of an
    earlier, larger one."""
    n, m, k0 = 3000, 30, 12
    kr = _kr(n, m)
    small = _kr(n, 2)
    A = _dense(n, 5)
    Am = _torch_dense_map(torch, kr, A)
    V = torch.zeros((m, n), dtype=torch.float64, device="cuda")
    H = np.zeros((m, m))
    f = torch.as_tensor(np.random.default_rng(6).standard_normal(n), device="cuda")
    kr.arnoldi(Am, V, H, f, 0, m)
    Q = np.linalg.qr(np.random.default_rng(7).standard_normal((m, m)))[0]
    Vo, fo = V.cpu().numpy().copy(), f.cpu().numpy().copy()
    Qo, Ho = Q.copy(), H.copy()
    kr.ira_restart(V, f, Q, H, k0)
    K.ira_restart(Vo, fo, Qo, Ho, k0)
    assert np.abs(V.cpu().numpy() - Vo).max() < 1e-12
    assert np.abs(f.cpu().numpy() - fo).max() < 1e-12
    small.close()
    kr.close()


def test_linearised_map_matches_the_reference_map(torch):
    """ns3d_map_linearised against the reference's own RK3_SSP_UV_RHS behind
    the reduced packing of NSCallMatrixVector_reduced (oracle/ref_harness.cu,
    the map the IRA benchmark's reference arm uses), on the same device
    vectors."""
    import ctypes

    from ns3dperiodic_b200 import Solver

    lib = os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref", "libns3d_ref.so")
    if not os.path.exists(lib):
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    from oracle.ref_lib import RefSolver

    g = O.Grid(16, 16, 16)
    Re = 40.0
    U = _kolmogorov(g, Re, 9)
    S = Solver(16, 16, 16)
    Ud = S.to_device(U)
    n = S.krylov_length
    kr = _kr(n, 2)
    A = kr.linearised_map(S, Ud, Re)
    ref = RefSolver(16, 16, 16)
    try:
        ref.set_u(U)
        fn = ref.lib.ref_map_linearised_reduced
        fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        fn.restype = None
        ctx = (ctypes.c_double * 2)(Re, 0.0)
        for seed in (1, 2):
            x = torch.as_tensor(np.random.default_rng(seed).standard_normal(n), device="cuda")
            y = torch.empty_like(x)
            yr = torch.empty_like(x)
            kr.apply(A, x, y)
            fn(ctypes.cast(ctx, ctypes.c_void_p), x.data_ptr(), yr.data_ptr())
            torch.cuda.synchronize()
            assert O.rel_l2(y.cpu().numpy(), yr.cpu().numpy()) < 1e-12
    finally:
        ref.close()
        kr.close()
        S.close()


def test_exponential_map_matches_the_reference_map(torch):
    """ns3d_map_exponential against the reference's own RK3_SSP_UV steps
    behind the reduced packing (oracle/ref_harness.cu
    ref_map_exponential_reduced, the map of the converged IRA benchmark's
    reference arm): two calls in a row, the base flow advancing with each,
    with the Kolmogorov forcing on both sides."""
    import ctypes

    from ns3dperiodic_b200 import Solver

    lib = os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref", "libns3d_ref.so")
    if not os.path.exists(lib):
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    from oracle.ref_lib import RefSolver

    g = O.Grid(16, 16, 16)
    Re, dt, steps = 40.0, 4e-3, 3
    U = _kolmogorov(g, Re, 9)
    F = O.kolmogorov_forcing(g)
    S = Solver(16, 16, 16)
    S.set_forcing(S.to_device(F))
    Ud, Vs = S.to_device(U), S.zeros()
    n = S.krylov_length
    kr = _kr(n, 2)
    A = kr.exponential_map(S, Ud, Vs, dt, Re, steps)
    ref = RefSolver(16, 16, 16)
    try:
        ref.set_u(U)
        ref.set_f(F)
        fn = ref.lib.ref_map_exponential_reduced
        fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        fn.restype = None
        ctx = (ctypes.c_double * 3)(Re, dt, float(steps))
        for seed in (1, 2):
            x = torch.as_tensor(np.random.default_rng(seed).standard_normal(n), device="cuda")
            y = torch.empty_like(x)
            yr = torch.empty_like(x)
            kr.apply(A, x, y)
            fn(ctypes.cast(ctx, ctypes.c_void_p), x.data_ptr(), yr.data_ptr())
            torch.cuda.synchronize()
            assert O.rel_l2(y.cpu().numpy(), yr.cpu().numpy()) < 1e-12
        assert O.rel_l2([u.cpu().numpy() for u in Ud], ref.get_u()) < 1e-12
    finally:
        ref.close()
        kr.close()
        S.close()
