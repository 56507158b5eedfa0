"""CPU oracle for the Krylov (Arnoldi / implicit-restart) path (TEST INFRASTRUCTURE).

This module is the checker, not the product.  Only ``tests/``,
``__graft_entry__.smoke()`` and the reference legs of ``bench.py`` may import
it.  It restates in numpy FP64, step by step, the reference's

* Arnoldi factorisation with classical Gram-Schmidt and iterative
  reorthogonalisation (Source/Arnoldi/Arnoldi_Driver.cu:29-120; tolerance
  5e-12 at :31, at most 13 passes at :60-72 and :97-115);
* implicit shifted QR on the Hessenberg matrix (Source/Arnoldi/QR_Shifts.cpp:
  7-72) with the Q factor of LAPACK's Householder QR (``dgeqrf`` + ``dormqr``,
  Source/Arnoldi/LAPACK_routines.cpp:289-345; numpy's ``qr`` is the same
  ``dgeqrf`` factorisation);
* shift selection (Source/Arnoldi/Select_Shifts.cpp:86-133);
* the restart update ``f = hl V q + ql f``, ``V = V Q`` with the trailing
  columns of Q reset to the identity
  (Source/Arnoldi/Implicit_restart_Arnoldi.cu:544-563);
* the 1-D periodic Laplacian test operator of the reference's Krylov
  self-test (Source/Arnoldi/Matrix_Vector_emulator.cu:10-36).

Layout follows the reference: ``V`` is n x m column-major (numpy arrays of
shape (m, n) here, row j = column j of V, which is the same memory), ``H``
is m x m column-major (numpy shape (m, m) indexed ``H[col, row]``; the
helpers take and return it as a normal row/column matrix ``Hm[row, col]``).

Parity status: pinned against the reference's own Krylov code built by
oracle/Makefile into oracle/_ref/libarnoldi_ref.so (Arnoldi_driver on a B200;
QR_shifts and select_shifts on the host with LAPACK from scipy's OpenBLAS),
through tests/golden/make_golden_krylov.py and tests/test_krylov_oracle.py.
"""
from __future__ import annotations

import numpy as np

ARNOLDI_TOL = 5.0e-12      # Source/Arnoldi/Arnoldi_Driver.cu:31
MAX_PASS_INDEX = 12        # "if(it>12) break" after the pass (:64,:109)
IM_EIG_TOL = 1.0e-15       # Source/Arnoldi/Macros.h:10


class ArnoldiBreakdown(RuntimeError):
    """||f|| < 1e-15 on entry with k == 0 (Arnoldi_Driver.cu:38-41)."""


def arnoldi_driver(Axb, V: np.ndarray, H: np.ndarray, f: np.ndarray, k: int, m: int,
                   tol: float = ARNOLDI_TOL) -> dict:
    """Extend an Arnoldi factorisation in place (Arnoldi_Driver.cu:29-120).

    ``V`` has shape (m, n) (row j is Krylov column j), ``H`` is a normal
    (m, m) matrix ``H[row, col]``, ``f`` the residual (n,).  ``Axb(v)``
    returns A v.  Returns statistics: reorthogonalisation passes per column
    and the number of columns that hit the pass limit.
    """
    passes = []
    failures = 0
    if k == 0:
        beta = float(np.sqrt(np.dot(f, f)))
        if beta < 1.0e-15:
            raise ArnoldiBreakdown("norm of the input vector ||f|| < 1e-15")
        v = f * (1.0 / beta)                       # Dcopy + Dscal(1/||f||)
        w = Axb(v)
        alpha = float(np.dot(v, w))
        f[:] = w - alpha * v                       # Dcopy + Daxpy(-alpha)
        c = 1.0
        it = 0
        while c > tol:                             # signed c, as in :60
            it += 1
            c = float(np.dot(v, f))
            f -= c * v
            alpha += c
            if it > MAX_PASS_INDEX:
                failures += 1
                break
        passes.append(it)
        H[0, 0] = alpha
        V[0, :] = v
    for j in range(k + 1, m):
        beta = float(np.sqrt(np.dot(f, f)))
        v = f * (1.0 / beta)
        H[j, j - 1] = beta
        V[j, :] = v
        w = Axb(v)
        Vj = V[: j + 1]
        h = np.zeros(m)
        h[: j + 1] = Vj @ w                        # Dgemv T, columns 0..j
        f[:] = w - Vj.T @ h[: j + 1]               # Dgemv N, alpha=-1, beta=1
        cn = 1.0
        it = 0
        while cn > tol:
            it += 1
            c = Vj @ f
            f -= Vj.T @ c
            h[: j + 1] += c
            cn = float(np.sqrt(np.dot(c, c)))
            if it > MAX_PASS_INDEX:
                failures += 1
                break
        passes.append(it)
        H[:, j] = h
    return {"passes": passes, "failures": failures}


def _householder_q(A: np.ndarray) -> np.ndarray:
    """Q factor of LAPACK's Householder QR (dgeqrf) of a square matrix."""
    q, _ = np.linalg.qr(A, mode="complete")
    return q


def _imag_exceeds(eig_im: float) -> bool:
    # QR_step tests abs() in double (QR_Shifts.cpp:9).
    return abs(eig_im) > IM_EIG_TOL


def _imag_exceeds_f32(eig_im: float) -> bool:
    # QR_shifts decrements j after testing fabsf(), i.e. in single precision
    # (QR_Shifts.cpp:63).
    return float(np.float32(abs(eig_im))) > IM_EIG_TOL


def qr_step(Qacc: np.ndarray, H: np.ndarray, eig: complex) -> tuple[np.ndarray, np.ndarray]:
    """One (double-)shift QR step (QR_Shifts.cpp:7-40); returns (Qacc Q, Q^T H Q)."""
    m = H.shape[0]
    er, ei = eig.real, eig.imag
    if _imag_exceeds(ei):
        H1 = H - er * np.eye(m)
        H1 = H1 @ H1 + (ei * ei) * np.eye(m)
    else:
        H1 = H - er * np.eye(m)
    Q = _householder_q(H1)
    Hn = (Q.T @ H) @ Q
    for j in range(m - 1):
        Hn[j + 2:, j] = 0.0                        # remove noise below the subdiagonal
    return Qacc @ Q, Hn


def qr_shifts(k: int, m: int, H: np.ndarray, eigs) -> tuple[np.ndarray, np.ndarray, int]:
    """QR_shifts (QR_Shifts.cpp:46-72): returns (Q, H_new, ko)."""
    Q = np.eye(m)
    Hn = np.array(H, dtype=np.float64, copy=True)
    j = m
    while j > k:
        e = complex(eigs[j - 1])
        Q, Hn = qr_step(Q, Hn, e)
        j -= 2 if _imag_exceeds_f32(e.imag) else 1
    return Q, Hn, j


def select_shifts(m: int, H: np.ndarray, which: str = "LR") -> tuple[np.ndarray, np.ndarray]:
    """select_shifts (Select_Shifts.cpp:86-133): eigenvalues of H sorted by
    'which' ("LR": largest real part first, "LM": largest modulus first) and
    the Ritz estimates |last component of each eigenvector|."""
    w, vecs = np.linalg.eig(np.asarray(H, dtype=np.complex128))
    if which == "LR":
        key = -w.real
    elif which == "LM":
        key = -np.abs(w)
    else:
        key = np.zeros(m)
    order = np.argsort(key, kind="stable")
    # zgeev normalises each eigenvector to unit 2-norm; so does numpy.
    ritz = np.abs(vecs[m - 1, order])
    return w[order], ritz


def ira_restart(V: np.ndarray, f: np.ndarray, Q: np.ndarray, H: np.ndarray, k0: int) -> float:
    """Restart update of Implicit_restart_Arnoldi.cu:544-563, in place.

    Returns ||f|| before the update (:547).  ``Q`` and ``H`` are normal
    (m, m) matrices; the columns k0..m-1 of Q are reset to the identity, as
    the reference does before forming V Q.
    """
    m = Q.shape[0]
    fnorm = float(np.sqrt(np.dot(f, f)))
    q = Q[:, k0].copy()
    hl = H[k0, k0 - 1]
    ql = Q[m - 1, k0 - 1]
    f[:] = hl * (V.T @ q) + ql * f                 # Dgemv N: alpha=hl, beta=ql
    Q[:, k0:] = np.eye(m)[:, k0:]
    V[:] = (V.T @ Q).T                             # Dgemm V Q
    return fnorm


def laplace1d(v: np.ndarray) -> np.ndarray:
    """The reference's Krylov test operator (Matrix_Vector_emulator.cu:10-20):
    w_i = v_{i+1} - 2 v_i + v_{i-1} periodic, then w_0 := 0."""
    w = np.roll(v, -1) - 2.0 * v + np.roll(v, 1)
    w[0] = 0.0
    return w


def arnoldi_residual(Axb, V: np.ndarray, H: np.ndarray, f: np.ndarray, m: int) -> float:
    """max |A V - V H - f e_m^T| relative to ||H||: the Arnoldi relation."""
    AV = np.stack([Axb(V[j]) for j in range(m)])           # rows = columns of A V
    VH = (V[:m].T @ H[:m, :m]).T
    R = AV - VH
    R[m - 1] -= f
    return float(np.abs(R).max() / max(np.abs(H).max(), 1.0))


# ---------------------------------------------------------------------------
# BiCGStab(L) and damped Newton (Source/Arnoldi/BiCGStabL.cu, Newton.cu)
# ---------------------------------------------------------------------------

def bicgstabl(Axb, x: np.ndarray, rhs: np.ndarray, L: int, tol: float, maxiter: int):
    """BiCGStabL (BiCGStabL.cu:18-185), x updated in place.

    Returns (flag, iterations, error) with the reference's flags: 0
    converged, 1 not converged, -1 rho = 0, -3 NaN; ``error`` is
    ||r||/||b|| and ``iterations`` the index of the last iteration run."""
    n = x.size
    r = [np.zeros(n) for _ in range(L + 1)]
    u = [np.zeros(n) for _ in range(L + 1)]
    tau = np.zeros(L * L)
    sigma = np.zeros(L + 1)
    gamma = np.zeros(L + 1)
    gamma_p = np.zeros(L + 1)
    gamma_pp = np.zeros(L + 1)
    flag = 1
    bnrm = float(np.sqrt(np.dot(rhs, rhs)))
    if bnrm < 1.0e-15:
        bnrm = 1.0
    r[0] = -(Axb(x) - rhs)                        # get_residualL: A x - b, then negated
    error = float(np.sqrt(np.dot(r[0], r[0]))) / bnrm
    if error < tol:
        flag = 0
    if np.isnan(error):
        flag = -3
    rt = r[0] * (1.0 / float(np.sqrt(np.dot(r[0], r[0])))) if flag == 1 else r[0].copy()
    rho, alpha, omega = 1.0, 0.0, 1.0
    it = 0
    if flag == 1:
        for it in range(maxiter):
            rho = -omega * rho
            for j in range(L):
                if rho == 0.0:
                    flag = -1
                    rho = 1.0
                rho1 = float(np.dot(r[j], rt))
                beta = alpha * rho1 / rho
                rho = rho1
                for i in range(j + 1):
                    u[i] = r[i] - beta * u[i]
                u[j + 1] = Axb(u[j])
                alpha = rho / float(np.dot(u[j + 1], rt))
                for i in range(j + 1):
                    r[i] = r[i] - alpha * u[i + 1]
                r[j + 1] = Axb(r[j])
                x += alpha * u[0]
            for j in range(1, L + 1):
                for i in range(1, j):
                    ij = (j - 1) * L + (i - 1)
                    tau[ij] = float(np.dot(r[j], r[i])) / sigma[i]
                    r[j] = r[j] - tau[ij] * r[i]
                sigma[j] = float(np.dot(r[j], r[j]))
                gamma_p[j] = float(np.dot(r[0], r[j])) / sigma[j]
            gamma[L] = gamma_p[L]
            omega = gamma[L]
            for j in range(L - 1, 0, -1):
                gamma[j] = gamma_p[j]
                for i in range(j + 1, L + 1):
                    gamma[j] -= tau[(i - 1) * L + (j - 1)] * gamma[i]
            for j in range(1, L):
                gamma_pp[j] = gamma[j + 1]
                for i in range(j + 1, L):
                    gamma_pp[j] += tau[(i - 1) * L + (j - 1)] * gamma[i + 1]
            x += gamma[1] * r[0]
            r[0] = r[0] - gamma_p[L] * r[L]
            u[0] = u[0] - gamma[L] * u[L]
            for j in range(1, L):
                x += gamma_pp[j] * r[j]
                r[0] = r[0] - gamma_p[j] * r[j]
                u[0] = u[0] - gamma[j] * u[j]
            error = float(np.sqrt(np.dot(r[0], r[0]))) / bnrm
            if error < tol:
                flag = 0
                break
            if error != error:
                flag = -3
                break
            if flag < 0:
                break
        else:
            it = maxiter
    return flag, it, error


def newton_initial_vector(n: int) -> np.ndarray:
    """set_initial_Krylov_vector_value_kernel (Arnoldi/cuda_supp.cu:451-465):
    zeros with 1.0, 1.5, 0.5, 1.0, 1.0 at indices 1, n/4, n/2, n-1, n-4 (every
    thread stores the fixed entries after its own zero, so the result is
    deterministic)."""
    d = np.zeros(n)
    d[1] = 1.0
    d[n // 4] = 1.5
    d[n // 2] = 0.5
    d[n - 1] = 1.0
    d[n - 4] = 1.0
    return d


def newton(jacobian, rhs_map, x: np.ndarray, tol: float, maxiter: int, tol_lin: float,
           iter_lin: int, L: int = 6, damping: float = 0.8):
    """Newton (Newton.cu:9-98), x updated in place.  ``rhs_map(x)`` returns
    F(x) and may record x as the point ``jacobian`` linearises about, as the
    reference's NSCallRHS_reduced does.  Returns (flag, iterations, tol_out,
    linsolve_flag): flag 0 converged, 1 not converged, 2 the linear solve
    failed (the reference exits there)."""
    n = x.size
    delta = newton_initial_vector(n)
    flag, ll, tol_out, lflag = 1, 0, tol, 0
    bn = rhs_map(x)
    if float(np.sqrt(np.dot(bn, bn))) < tol:
        return 0, 0, tol, 0
    for ll in range(maxiter):
        bn = -rhs_map(x)
        lflag, _, _ = bicgstabl(jacobian, delta, bn, L, tol_lin, iter_lin)
        if lflag != 0:
            return 2, ll, tol_out, lflag
        x += damping * delta
        tol_newton = float(np.sqrt(np.dot(delta, delta)))
        norm_rhs = float(np.sqrt(np.dot(bn, bn)))
        if norm_rhs < tol and ll > 2:
            return 0, ll, tol_newton, 0
    else:
        ll = maxiter
    return flag, ll, tol_out, lflag


# ---------------------------------------------------------------------------
# Final stage of the implicit restart and the matrix-exponent driver
# (Source/Arnoldi/Implicit_restart_Arnoldi.cu:255-742)
# ---------------------------------------------------------------------------

def _sorted_eig(R: np.ndarray, which: str):
    """MatrixComplexEigensystem + get_sorted_index: eigenpairs of R (unit
    eigenvectors, zgeev) sorted by 'which'."""
    w, Y = np.linalg.eig(np.asarray(R, dtype=np.complex128))
    key = -w.real if which == "LR" else -np.abs(w)
    order = np.argsort(key, kind="stable")
    return w[order], Y[:, order]


def schur_basis(V: np.ndarray, H: np.ndarray, k: int) -> np.ndarray:
    """Schur_Hessinberg_matrix + V1 = V Q_Schur (Implicit_restart_Arnoldi.cu:
    616-632): the real Schur vectors Z of H[:k, :k] (dhseqr; scipy's LAPACK
    here) and the rows of V1 = (Z^T V[:k])."""
    from scipy.linalg import schur

    _, Z = schur(np.asarray(H[:k, :k], dtype=np.float64), output="real")
    return Z.T @ V[:k]


def eigensystem_no_rotation(Axb, V1: np.ndarray, which: str = "LR"):
    """compute_eigensystem_of_original_mapping_no_rotation
    (Implicit_restart_Arnoldi.cu:255-330): R = V1^T A V1 (R[i, j] =
    v1_i . A v1_j), residuals ||A v1_j - sum_i v1_i R[i, j]||, eigenpairs of R
    sorted by 'which', eigenvectors V1 y.  Returns (w, X rows, residuals)."""
    AV = np.stack([Axb(v) for v in V1])
    R = V1 @ AV.T
    res = np.linalg.norm(AV - R.T @ V1, axis=1)
    w, Y = _sorted_eig(R, which)
    return w, Y.T @ V1, res


def eigensystem_rotation(Axb, V1: np.ndarray, which: str = "LR"):
    """compute_eigensystem_of_original_mapping_rotation
    (Implicit_restart_Arnoldi.cu:335-434): V1 holds k doubled Schur vectors;
    VR, VI are their halves, R = VR^T A VR + VI^T A VI with the original map
    A (half length), the residuals ||A vr_j - VR R e_j|| and
    ||A vi_j - VI R e_j||, eigenpairs of R sorted by 'which' and the
    eigenvectors (VR + VI) y.  Returns (w, X rows, res_real, res_imag)."""
    n = V1.shape[1] // 2
    VR, VI = V1[:, :n], V1[:, n:]
    AVR = np.stack([Axb(v) for v in VR])
    AVI = np.stack([Axb(v) for v in VI])
    R = VR @ AVR.T + VI @ AVI.T
    res_r = np.linalg.norm(AVR - R.T @ VR, axis=1)
    res_i = np.linalg.norm(AVI - R.T @ VI, axis=1)
    w, Y = _sorted_eig(R, which)
    return w, Y.T @ (VR + VI), res_r, res_i


def ira_matrix_exponent(Axb_invert, Axb, n_rot: int, k: int, m: int, which: str = "LR",
                        which_exponent: str = "LM", tol: float = 5.0e-8, max_iter: int = 3000,
                        rotated: bool = False, f0: np.ndarray | None = None, seed: int = 0):
    """Implicit_restart_Arnoldi_GPU_data_Matrix_Exponent
    (Implicit_restart_Arnoldi.cu:456-742): the restart loop (:531-581) on
    ``Axb_invert`` over vectors of length n_rot ordered by 'which_exponent',
    then the final stage on the original map ``Axb``.  The start vector is
    N(0, 2) (rand_normal(0, 2), :485-488) from a seeded generator.  Returns a
    dict like the GPU path's."""
    f = (np.random.default_rng(seed).normal(0.0, 2.0, n_rot) if f0 is None
         else np.array(f0, dtype=np.float64))
    V = np.zeros((m, n_rot))
    H = np.zeros((m, m))
    k0, it, ritz_norm = 1, 0, 1.0
    eig = np.zeros(m, dtype=np.complex128)
    while it < max_iter and ritz_norm > tol:
        it += 1
        arnoldi_driver(Axb_invert, V, H, f, k0 - 1, m)
        eig, ritz = select_shifts(m, H, which_exponent)
        Q, H, k0 = qr_shifts(k, m, H, eig)
        fnorm = ira_restart(V, f, Q, H, k0)
        ritz = ritz * fnorm
        ritz_norm = float(np.max(np.abs(ritz[:k0]).astype(np.float32)))
    V1 = schur_basis(V, H, k)
    if rotated:
        w, X, rr, ri = eigensystem_rotation(Axb, V1, which)
    else:
        w, X, rr = eigensystem_no_rotation(Axb, V1, which)
        ri = np.zeros_like(rr)
    return {"eigenvalues": w, "eigenvectors": X, "residual_real": rr, "residual_imag": ri,
            "ritz_norm": ritz_norm, "iterations": it, "eigenvalues_invert": eig, "V": V, "H": H}
