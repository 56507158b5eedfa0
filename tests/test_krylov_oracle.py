"""Krylov oracle and host-side Krylov code against the reference's own
outputs (tests/golden/krylov_*.npz, made by tests/golden/make_golden_krylov.py
from the reference's Source/Arnoldi build).  No GPU needed.

The QR-shift comparison covers the parts of Q and H that are determined by
the input: the leading ko columns of Q, the leading ko x ko block of H and
H(ko, ko-1).  The trailing columns belong to the subspace the exact shifts
deflate; there the explicit shifted QR is forward-unstable and two LAPACK
builds (or the reference run twice with different BLAS) disagree at O(1e-1),
so only their structure is checked.
"""
import os

import numpy as np
import pytest

from oracle import krylov_oracle as K

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
QR_TOL = 1e-12          # leading Q columns / H block, absolute (entries are O(1))


def _qr_cases():
    d = np.load(os.path.join(GOLDEN, "krylov_qr.npz"))
    for i in range(int(d["ncases"])):
        yield i, {k[len(f"c{i}_"):]: d[k] for k in d.files if k.startswith(f"c{i}_")}


def _check_qr(Q, H, ko, case):
    n, m, k, seed, ko_ref = (int(x) for x in case["meta"])
    assert ko == ko_ref
    assert np.abs(Q[:, :ko] - case["Q"][:, :ko]).max() < QR_TOL
    assert np.abs(H[:ko, :ko] - case["H_out"][:ko, :ko]).max() < QR_TOL
    assert abs(H[ko, ko - 1] - case["H_out"][ko, ko - 1]) < QR_TOL
    # structure of the whole result
    assert np.abs(Q.T @ Q - np.eye(m)).max() < 1e-13
    assert np.abs(np.tril(H, -2)).max() == 0.0


@pytest.mark.parametrize("i", range(6))
def test_oracle_qr_shifts_matches_reference(i):
    case = dict(_qr_cases())[i]
    eig = case["eig_re"] + 1j * case["eig_im"]
    Q, H, ko = K.qr_shifts(int(case["meta"][2]), int(case["meta"][1]), case["H_in"], eig)
    _check_qr(Q, H, ko, case)


@pytest.mark.parametrize("i", range(6))
def test_library_qr_shifts_matches_reference(i):
    """ns3d_qr_shifts is host code of the CUDA library: callable without a GPU."""
    from ns3dperiodic_b200 import krylov as KR

    case = dict(_qr_cases())[i]
    eig = case["eig_re"] + 1j * case["eig_im"]
    Q, H, ko = KR.qr_shifts(int(case["meta"][2]), case["H_in"], eig)
    _check_qr(Q, H, ko, case)


def test_select_shifts_match_reference():
    from ns3dperiodic_b200 import krylov as KR

    for _, case in _qr_cases():
        m = int(case["meta"][1])
        for fn in (lambda H: K.select_shifts(m, H, "LR"), lambda H: KR.select_shifts(H, "LR")):
            e, r = fn(case["H_in"])
            assert np.abs(e.real - case["eig_re"]).max() < 1e-13
            assert np.abs(e.imag - case["eig_im"]).max() < 1e-13
            assert np.abs(r - case["ritz"]).max() < 1e-12


def test_qr_shift_count_follows_conjugate_pairs():
    """A complex shift consumes two eigenvalues; the last case ends at k - 1."""
    cases = dict(_qr_cases())
    n, m, k, seed, ko = (int(x) for x in cases[5]["meta"])
    assert ko == k - 1
    assert abs(cases[5]["eig_im"][k - 1]) > 1e-15


def _arnoldi_golden():
    path = os.path.join(GOLDEN, "krylov_arnoldi.npz")
    if not os.path.exists(path):
        pytest.fail("tests/golden/krylov_arnoldi.npz is missing (make_golden_krylov.py)")
    return np.load(path)


def _dense(n, seed):
    return np.random.default_rng(seed).standard_normal((n, n)) / np.sqrt(n)


@pytest.mark.parametrize("name", ["laplace", "dense"])
def test_oracle_arnoldi_matches_reference(name):
    d = _arnoldi_golden()
    n, m, kc, seed = (int(x) for x in d[f"{name}_meta"])
    Axb = K.laplace1d if name == "laplace" else (lambda v, A=_dense(n, seed): A @ v)
    V = np.zeros((m, n))
    H = np.zeros((m, m))
    f = d[f"{name}_f0"].copy()
    K.arnoldi_driver(Axb, V, H, f, 0, m)
    sc = np.abs(d[f"{name}_H"]).max()
    assert np.abs(H - d[f"{name}_H"]).max() < 1e-12 * sc
    assert np.abs(V - d[f"{name}_V"]).max() < 1e-11
    assert np.abs(f - d[f"{name}_f"]).max() < 1e-11 * max(1.0, np.abs(d[f"{name}_f"]).max())
    # continuation from column kc
    V = d[f"{name}_cont_V_in"].copy()
    H = d[f"{name}_cont_H_in"].copy()
    f = d[f"{name}_cont_f_in"].copy()
    K.arnoldi_driver(Axb, V, H, f, kc, m)
    assert np.abs(H - d[f"{name}_cont_H"]).max() < 1e-12 * sc
    assert np.abs(V - d[f"{name}_cont_V"]).max() < 1e-11


def test_oracle_laplace_operator_matches_reference():
    d = _arnoldi_golden()
    np.testing.assert_array_equal(K.laplace1d(d["laplace_apply_in"]), d["laplace_apply_out"])


def test_oracle_arnoldi_relation_and_orthogonality():
    rng = np.random.default_rng(5)
    n, m = 400, 24
    A = rng.standard_normal((n, n)) / np.sqrt(n)
    V = np.zeros((m, n))
    H = np.zeros((m, m))
    f = rng.standard_normal(n)
    st = K.arnoldi_driver(lambda v: A @ v, V, H, f, 0, m)
    assert st["failures"] == 0 and max(st["passes"]) <= 3
    assert np.abs(V @ V.T - np.eye(m)).max() < 1e-13
    assert K.arnoldi_residual(lambda v: A @ v, V, H, f, m) < 1e-13
    assert np.abs(V @ f).max() < 1e-12 * np.linalg.norm(f)
    assert np.abs(np.tril(H, -2)).max() == 0.0


def test_oracle_restart_keeps_a_k_step_factorisation():
    """After QR shifts + restart, A V_k = V_k H_k + f e_k^T holds for the k0
    leading columns (Sorensen's implicit restart)."""
    rng = np.random.default_rng(6)
    n, m, k = 300, 20, 6
    X = np.eye(n) + 0.1 * rng.standard_normal((n, n))
    A = X @ np.diag(np.linspace(1.0, 0.05, n)) @ np.linalg.inv(X)
    V = np.zeros((m, n))
    H = np.zeros((m, m))
    f = rng.standard_normal(n)
    K.arnoldi_driver(lambda v: A @ v, V, H, f, 0, m)
    eig, _ = K.select_shifts(m, H, "LR")
    Q, Hn, k0 = K.qr_shifts(k, m, H, eig)
    K.ira_restart(V, f, Q, Hn, k0)
    Ax = lambda v: A @ v  # noqa: E731
    Vk, Hk = V[:k0], Hn[:k0, :k0]
    R = np.stack([Ax(Vk[j]) for j in range(k0)]) - (Vk.T @ Hk).T
    R[k0 - 1] -= f
    assert np.abs(R).max() < 1e-8
    assert np.abs(Vk @ Vk.T - np.eye(k0)).max() < 1e-12


def test_oracle_arnoldi_rejects_zero_start():
    with pytest.raises(K.ArnoldiBreakdown):
        K.arnoldi_driver(K.laplace1d, np.zeros((4, 10)), np.zeros((4, 4)), np.zeros(10), 0, 4)


def _linsolve_golden():
    path = os.path.join(GOLDEN, "krylov_linsolve.npz")
    if not os.path.exists(path):
        pytest.fail("tests/golden/krylov_linsolve.npz is missing (make_golden_krylov.py)")
    return np.load(path)


def _lin_matrix(n, seed, diag, scale):
    rng = np.random.default_rng(seed)
    return diag * np.eye(n) + scale * rng.standard_normal((n, n)) / np.sqrt(n)


@pytest.mark.parametrize("idx", range(3))
def test_oracle_bicgstabl_matches_reference(idx):
    d = _linsolve_golden()
    n, L, seed, flag, it = (int(v) for v in d[f"bicg{idx}_meta"])
    A = _lin_matrix(n, seed, 2.0, 0.5)
    x = np.zeros(n)
    fl, its, err = K.bicgstabl(lambda v: A @ v, x, d[f"bicg{idx}_b"], L, 1e-10, 200)
    assert (fl, its) == (flag, it)
    assert abs(err - float(d[f"bicg{idx}_err"][0])) < 1e-3 * float(d[f"bicg{idx}_err"][0])
    assert np.abs(x - d[f"bicg{idx}_x"]).max() < 1e-10 * np.abs(d[f"bicg{idx}_x"]).max()


def test_oracle_newton_matches_reference():
    d = _linsolve_golden()
    n, seed, flag, it = (int(v) for v in d["newton_meta"])
    c, tol_out = (float(v) for v in d["newton_c_tol"])
    A = _lin_matrix(n, seed, 3.0, 0.3)
    b = d["newton_b"]
    st = {"base": np.zeros(n)}

    def F(x):
        st["base"] = x.copy()
        return A @ x + c * x ** 3 - b

    x = np.zeros(n)
    fl, its, t, lf = K.newton(lambda v: A @ v + 3 * c * st["base"] ** 2 * v, F, x, 1e-9, 60,
                              1e-11, 200)
    assert (fl, its, lf) == (flag, it, 0)
    assert abs(t - tol_out) < 1e-6 * tol_out + 1e-14
    assert np.abs(x - d["newton_x"]).max() < 1e-10 * np.abs(d["newton_x"]).max()


def test_oracle_bicgstabl_solves_and_flags():
    rng = np.random.default_rng(9)
    n = 150
    A = 2.0 * np.eye(n) + 0.5 * rng.standard_normal((n, n)) / np.sqrt(n)
    b = rng.standard_normal(n)
    for L in (1, 3, 6):
        x = np.zeros(n)
        fl, its, err = K.bicgstabl(lambda v: A @ v, x, b, L, 1e-12, 300)
        assert fl == 0 and err < 1e-12
        assert np.abs(A @ x - b).max() < 1e-10
    # already solved: flag 0 without iterating
    x = np.linalg.solve(A, b)
    fl, its, err = K.bicgstabl(lambda v: A @ v, x, b, 2, 1e-8, 10)
    assert fl == 0 and its == 0
    # NaN in the map: flag -3
    fl, its, err = K.bicgstabl(lambda v: v * np.nan, np.zeros(n), b, 2, 1e-8, 10)
    assert fl == -3
