"""Oracle of the shift-invert (matrix-exponent) implicit restart against the
reference's own Implicit_restart_Arnoldi_GPU_data_Matrix_Exponent
(tests/golden/krylov_shift_invert.npz, made by
tests/golden/make_golden_shift_invert.py from the reference's Source/Arnoldi
build on a B200), and the oracle's shifted maps against their definition.
No GPU needed.

The reference never fills its eigenvalue argument, so its eigenvalues are
the Rayleigh quotients of the eigenvectors it returns; converged eigenpairs
agree to 1e-8 (Ritz tolerance 5e-8 on a well-conditioned spectrum).
"""
import math
import os

import numpy as np
import pytest

from oracle import krylov_oracle as K
from oracle import ns3d_oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


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
def test_oracle_driver_matches_reference_golden(tag):
    z = np.load(os.path.join(GOLDEN, "krylov_shift_invert.npz"))
    A, Minv = z["A"], z[f"Minv_{tag}"]
    k, m, tol = int(z["k"]), int(z["m"]), float(z["tol"])
    o = K.ira_matrix_exponent(lambda v: Minv @ v, lambda v: A @ v, Minv.shape[0], k, m, "LR",
                              "LM", tol, 200, rotated=(tag == "rotated"), seed=1)
    assert o["ritz_norm"] <= tol
    lam_ref, res_ref = _rayleigh(A, z[f"vec_re_{tag}"] + 1j * z[f"vec_im_{tag}"])
    assert res_ref.max() < 1e-8
    assert float(z[f"ritz_{tag}"]) <= tol
    w = o["eigenvalues"]
    assert _set_distance(w, lam_ref) < 1e-8
    # the eigenvalues of A nearest the shift sigma (e^{i theta})
    ev = np.linalg.eigvals(A)
    s = float(z["sigma"]) * (complex(math.cos(float(z["theta"])), math.sin(float(z["theta"])))
                             if tag == "rotated" else 1.0)
    near = sorted(ev, key=lambda e: abs(e - s))[:2]
    for e in near:
        assert np.abs(w - e).min() < 1e-8
    X = o["eigenvectors"]
    for i in range(k):
        assert np.linalg.norm(A @ X[i] - w[i] * X[i]) < 1e-8 * np.linalg.norm(X[i])


def test_eigensystem_rotation_reduces_to_the_plain_stage():
    """With a zero imaginary half the rotated final stage is the plain one."""
    rng = np.random.default_rng(2)
    n, k = 30, 4
    A = rng.standard_normal((n, n))
    V1 = np.linalg.qr(rng.standard_normal((n, k)))[0].T
    w, X, r = K.eigensystem_no_rotation(lambda v: A @ v, V1, "LR")
    w2, X2, rr, ri = K.eigensystem_rotation(lambda v: A @ v,
                                            np.concatenate([V1, np.zeros_like(V1)], axis=1), "LR")
    assert np.abs(w - w2).max() < 1e-14
    assert np.abs(X - X2).max() < 1e-14
    assert np.abs(r - rr).max() < 1e-14 and ri.max() == 0.0


def test_oracle_rotated_map_is_the_complex_shift():
    g = O.Grid(8, 8, 8)
    Re, dt, steps, sigma, theta = 20.0, 0.02, 2, 1.05, 0.05
    U, _ = O.kolmogorov_state(g, Re, 1, rel_amp=1e-2)
    n = 3 * (g.Nx * g.Ny * g.Mz - 1)
    rng = np.random.default_rng(3)
    xr, xi = rng.standard_normal(n), rng.standard_normal(n)
    er = O.exponential_shifted_reduced(g, U, xr, dt, Re, steps, 0.0)
    ei = O.exponential_shifted_reduced(g, U, xi, dt, Re, steps, 0.0)
    s = sigma * complex(math.cos(theta), math.sin(theta))
    z = er + 1j * ei - s * (xr + 1j * xi)
    out = O.exponential_rotated_reduced(g, U, np.concatenate([xr, xi]), dt, Re, steps, sigma,
                                        theta)
    assert np.abs(out[:n] - z.real).max() < 1e-13 * np.abs(z).max()
    assert np.abs(out[n:] - z.imag).max() < 1e-13 * np.abs(z).max()
    # E is linear and the shift is -sigma * x
    y = O.exponential_shifted_reduced(g, U, 2.0 * xr, dt, Re, steps, sigma)
    assert np.abs(y - 2.0 * (er - sigma * xr)).max() < 1e-12 * np.abs(y).max()


def test_reference_library_exports_the_driver():
    import ctypes

    lib = os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref", "libarnoldi_ref.so")
    if not os.path.exists(lib):
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    assert hasattr(ctypes.CDLL(lib), "ref_ira_matrix_exponent_dense")
