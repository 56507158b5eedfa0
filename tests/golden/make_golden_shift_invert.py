"""Generate golden vectors for the shift-invert (matrix-exponent) implicit
restart from the reference's own code.

oracle/Makefile builds the reference's Source/Arnoldi sources, unmodified,
into oracle/_ref/libarnoldi_ref.so, including
Implicit_restart_Arnoldi_GPU_data_Matrix_Exponent
(Implicit_restart_Arnoldi.cu:456-742).  This script runs it (cuBLAS, needs a
GPU) with dense operators standing in for the Navier-Stokes maps: the
original map is a seeded non-normal matrix A with known eigenvalues, the
shift-invert map is (A - sigma)^{-1} (no rotation) or the real form of
(A - sigma e^{i theta})^{-1} on vectors of length 2n (rotation), with the
shift main uses (sigma = 1.05, theta = 0.05, Source/NS3D_periodic.cu:
1652-1653).  It writes tests/golden/krylov_shift_invert.npz with the
operators and the reference's eigenvectors (its eigenvalue argument is never
filled; the reference prints them).

Made with:

    make -C oracle && python tests/golden/make_golden_shift_invert.py --out tests/golden

The reference seeds its start vector from the clock and writes H_pre.dat,
H_Schur.dat and Q_Schur.dat into the working directory; the script runs it
in a temporary directory.  Converged eigenpairs do not depend on the start
vector beyond the tolerance.
"""
from __future__ import annotations

import argparse
import ctypes
import math
import os
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
LIB = os.path.join(ROOT, "oracle", "_ref", "libarnoldi_ref.so")
_dp = ctypes.POINTER(ctypes.c_double)

SIGMA, THETA = 1.05, 0.05
N, K, M = 48, 6, 20
TOL, MAX_ITER = 5.0e-8, 200


def _p(a):
    return a.ctypes.data_as(_dp)


def operator(n: int, seed: int) -> np.ndarray:
    """Dense non-normal n x n matrix: real eigenvalues spread over [-3, 0.4]
    and complex pairs around the shift, X = I + N(0,1)/sqrt(n)."""
    rng = np.random.default_rng(seed)
    pairs = [(1.1, 0.05), (0.9, 0.3), (1.0, 0.6), (0.5, 0.1), (0.2, 1.0), (-0.5, 2.0)]
    D = np.zeros((n, n))
    nreal = n - 2 * len(pairs)
    D[:nreal, :nreal] = np.diag(np.linspace(-3.0, 0.4, nreal))
    i = nreal
    for a, b in pairs:
        D[i:i + 2, i:i + 2] = [[a, b], [-b, a]]
        i += 2
    X = rng.standard_normal((n, n)) / math.sqrt(n) + np.eye(n)
    return X @ D @ np.linalg.inv(X)


def shift_invert(A: np.ndarray, rotated: bool) -> np.ndarray:
    n = A.shape[0]
    I = np.eye(n)
    if not rotated:
        return np.linalg.inv(A - SIGMA * I)
    sr, si = SIGMA * math.cos(THETA), SIGMA * math.sin(THETA)
    return np.linalg.inv(np.block([[A - sr * I, si * I], [-si * I, A - sr * I]]))


def run_reference(lib, A, Minv, rotated: bool):
    n = A.shape[0]
    Af = np.asfortranarray(A)
    Mf = np.asfortranarray(Minv)
    vr = np.zeros((K, n))
    vi = np.zeros((K, n))
    ritz = ctypes.c_double(0.0)
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.chdir(tmp)
        try:
            rc = lib.ref_ira_matrix_exponent_dense(n, int(rotated), _p(Mf), _p(Af), K, M,
                                                   ctypes.c_double(TOL), MAX_ITER, _p(vr),
                                                   _p(vi), ctypes.byref(ritz))
        finally:
            os.chdir(cwd)
    if rc != 0:
        raise RuntimeError(f"ref_ira_matrix_exponent_dense failed: {rc}")
    return vr, vi, ritz.value


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    args = ap.parse_args()
    lib = ctypes.CDLL(LIB)
    lib.ref_ira_matrix_exponent_dense.restype = ctypes.c_int
    A = operator(N, 11)
    out = {"A": A, "sigma": SIGMA, "theta": THETA, "k": K, "m": M, "tol": TOL}
    for tag, rotated in (("plain", False), ("rotated", True)):
        Minv = shift_invert(A, rotated)
        vr, vi, ritz = run_reference(lib, A, Minv, rotated)
        out[f"Minv_{tag}"] = Minv
        out[f"vec_re_{tag}"] = vr
        out[f"vec_im_{tag}"] = vi
        out[f"ritz_{tag}"] = ritz
        X = vr + 1j * vi
        lam = np.array([np.vdot(x, A @ x) / np.vdot(x, x) for x in X])
        res = [np.linalg.norm(A @ x - l * x) / np.linalg.norm(x) for x, l in zip(X, lam)]
        print(tag, "ritz", ritz, "eigenvalues", np.round(lam, 10), "residuals", res)
    path = os.path.join(args.out, "krylov_shift_invert.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)


if __name__ == "__main__":
    main()
