"""Generate golden vectors for the Krylov path from the reference's own code.

oracle/Makefile builds the reference's Source/Arnoldi sources, unmodified,
into oracle/_ref/libarnoldi_ref.so.  This script runs them on seeded inputs
and writes tests/golden/krylov_*.npz:

* ``krylov_qr.npz``     QR_shifts and select_shifts (host code; LAPACK from
                        scipy's OpenBLAS) on Hessenberg matrices of seeded
                        operators with well-separated spectra;
* ``krylov_arnoldi.npz`` Arnoldi_driver (cuBLAS, needs a GPU) with the
                        reference's 1-D periodic Laplacian and with a dense
                        seeded matrix, started from k = 0 and continued from
                        k > 0, plus one application of the Laplacian.

Made with:

    make -C oracle && python tests/golden/make_golden_krylov.py --out tests/golden

* ``krylov_linsolve.npz`` BiCGStabL (L = 1, 2, 6) on a seeded dense system and
                        Newton on a seeded cubic problem F(x) = A x + c x^3 - b
                        (cuBLAS, needs a GPU).

(``--host-only`` writes only krylov_qr.npz, without a GPU; ``--arnoldi-only``
writes only krylov_arnoldi.npz; ``--linsolve-only`` only krylov_linsolve.npz.)
"""
from __future__ import annotations

import argparse
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import krylov_oracle as K  # noqa: E402

LIB = os.path.join(ROOT, "oracle", "_ref", "libarnoldi_ref.so")
_dp = ctypes.POINTER(ctypes.c_double)


def _p(a):
    return a.ctypes.data_as(_dp)


def seeded_operator(n: int, seed: int, pairs: int = 5) -> np.ndarray:
    """Dense non-normal n x n matrix with eigenvalues 1 .. 0.05 and `pairs`
    complex-conjugate pairs, made well conditioned (X = I + 0.1 N(0,1))."""
    rng = np.random.default_rng(seed)
    lam = np.linspace(1.0, 0.05, n)
    D = np.diag(lam)
    for i in range(0, 2 * pairs, 2):
        b = 0.1 * (i + 1)
        D[i:i + 2, i:i + 2] = [[lam[i], b], [-b, lam[i]]]
    X = rng.standard_normal((n, n)) * 0.1 + np.eye(n)
    return X @ D @ np.linalg.inv(X)


def dense_matrix(n: int, seed: int) -> np.ndarray:
    """Seeded dense matrix used for the Arnoldi golden (scaled Gaussian)."""
    return np.random.default_rng(seed).standard_normal((n, n)) / np.sqrt(n)


QR_CASES = [  # (n, m, k, seed); the last one ends at ko = k - 1 (a complex pair straddles k)
    (200, 12, 4, 3),
    (300, 30, 10, 3),
    (240, 16, 6, 10),
    (240, 20, 8, 14),
    (300, 24, 12, 12),
    (160, 10, 3, 12),
]

ARNOLDI_CASES = {  # name: (operator, n, m, k_continue, seed)
    "laplace": ("laplace", 1000, 12, 5, 21),
    "dense": ("dense", 300, 16, 6, 22),
}


def make_qr(lib) -> dict:
    out = {}
    for idx, (n, m, k, seed) in enumerate(QR_CASES):
        A = seeded_operator(n, seed)
        V = np.zeros((m, n))
        H = np.zeros((m, m))
        f = np.random.default_rng(seed + 100).standard_normal(n)
        K.arnoldi_driver(lambda v: A @ v, V, H, f, 0, m)
        Hf = np.asfortranarray(H)
        er, ei, ritz = np.zeros(m), np.zeros(m), np.zeros(m)
        lib.ref_select_shifts(m, _p(Hf.copy(order="F")), b"LR", _p(er), _p(ei), _p(ritz))
        Q = np.zeros((m, m), order="F")
        Hout = Hf.copy(order="F")
        ko = ctypes.c_int(0)
        lib.ref_qr_shifts(k, m, _p(Q), _p(Hout), _p(er), _p(ei), ctypes.byref(ko))
        # keep only cases whose leading part is well conditioned: the oracle
        # (numpy LAPACK) must agree with the reference there
        Qo, Ho, kk = K.qr_shifts(k, m, H, er + 1j * ei)
        assert kk == ko.value
        dq = np.abs(Qo[:, :kk] - Q[:, :kk]).max()
        assert dq < 1e-12, (idx, dq)
        pre = f"c{idx}_"
        out[pre + "H_in"] = H
        out[pre + "eig_re"] = er
        out[pre + "eig_im"] = ei
        out[pre + "ritz"] = ritz
        out[pre + "Q"] = np.ascontiguousarray(Q)
        out[pre + "H_out"] = np.ascontiguousarray(Hout)
        out[pre + "meta"] = np.array([n, m, k, seed, ko.value])
    out["ncases"] = np.array(len(QR_CASES))
    return out


def make_arnoldi(lib) -> dict:
    out = {}
    for name, (op, n, m, kc, seed) in ARNOLDI_CASES.items():
        rng = np.random.default_rng(seed)
        f0 = rng.standard_normal(n)
        V = np.zeros((m, n))
        H = np.zeros((m, m), order="F")
        f = f0.copy()
        if op == "laplace":
            rc = lib.ref_arnoldi_laplace(n, m, 0, _p(V), _p(H), _p(f))
        else:
            A = np.asfortranarray(dense_matrix(n, seed))
            rc = lib.ref_arnoldi_dense(n, m, 0, _p(A), _p(V), _p(H), _p(f))
        assert rc == 0, rc
        out[f"{name}_f0"] = f0
        out[f"{name}_V"] = V.copy()
        out[f"{name}_H"] = np.ascontiguousarray(H)
        out[f"{name}_f"] = f.copy()
        # continuation from column kc: keep V(:, :kc+1), H(:kc+1, :kc+1), f
        V2 = V.copy()
        V2[kc + 1:] = 0.0
        H2 = np.asfortranarray(np.array(H))
        H2[:, kc + 1:] = 0.0
        H2[kc + 1:, :] = 0.0
        fc = np.random.default_rng(seed + 1).standard_normal(n)
        out[f"{name}_cont_V_in"] = V2.copy()
        out[f"{name}_cont_H_in"] = np.ascontiguousarray(H2)
        out[f"{name}_cont_f_in"] = fc.copy()
        if op == "laplace":
            rc = lib.ref_arnoldi_laplace(n, m, kc, _p(V2), _p(H2), _p(fc))
        else:
            rc = lib.ref_arnoldi_dense(n, m, kc, _p(A), _p(V2), _p(H2), _p(fc))
        assert rc == 0, rc
        out[f"{name}_cont_V"] = V2
        out[f"{name}_cont_H"] = np.ascontiguousarray(H2)
        out[f"{name}_cont_f"] = fc
        out[f"{name}_meta"] = np.array([n, m, kc, seed])
    x = np.random.default_rng(31).standard_normal(777)
    y = np.zeros_like(x)
    assert lib.ref_laplace_apply(x.size, _p(x), _p(y)) == 0
    out["laplace_apply_in"] = x
    out["laplace_apply_out"] = y
    return out


def linsolve_matrix(n: int, seed: int, diag: float, scale: float) -> np.ndarray:
    """Seeded non-symmetric matrix diag*I + scale*N(0,1)/sqrt(n)."""
    rng = np.random.default_rng(seed)
    return diag * np.eye(n) + scale * rng.standard_normal((n, n)) / np.sqrt(n)


BICG_CASES = [(300, L, 41) for L in (1, 2, 6)]  # (n, L, seed): tol 1e-10, 200 iterations
NEWTON_CASE = (200, 42, 0.1)                     # (n, seed, c): tol 1e-9, 60 iterations


def make_linsolve(lib) -> dict:
    out = {}
    for idx, (n, L, seed) in enumerate(BICG_CASES):
        A = np.asfortranarray(linsolve_matrix(n, seed, 2.0, 0.5))
        b = np.random.default_rng(seed + 1).standard_normal(n)
        x = np.zeros(n)
        tol = np.array([1e-10])
        it = ctypes.c_int(200)
        flag = lib.ref_bicgstabl_dense(n, L, _p(A), _p(x), _p(b), _p(tol), ctypes.byref(it))
        assert flag == 0, flag
        pre = f"bicg{idx}_"
        out[pre + "b"] = b
        out[pre + "x"] = x
        out[pre + "meta"] = np.array([n, L, seed, flag, it.value])
        out[pre + "err"] = tol
    n, seed, c = NEWTON_CASE
    A = np.asfortranarray(linsolve_matrix(n, seed, 3.0, 0.3))
    b = np.random.default_rng(seed + 1).standard_normal(n)
    x = np.zeros(n)
    tol = np.array([1e-9])
    it = ctypes.c_int(60)
    flag = lib.ref_newton_cubic(n, _p(A), _p(b), c, _p(x), _p(tol), ctypes.byref(it), 1e-11, 200)
    assert flag == 0, flag
    out["newton_b"] = b
    out["newton_x"] = x
    out["newton_meta"] = np.array([n, seed, flag, it.value])
    out["newton_c_tol"] = np.array([c, tol[0]])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    ap.add_argument("--host-only", action="store_true")
    ap.add_argument("--arnoldi-only", action="store_true")
    ap.add_argument("--linsolve-only", action="store_true")
    a = ap.parse_args()
    lib = ctypes.CDLL(LIB)
    lib.ref_select_shifts.argtypes = [ctypes.c_int, _dp, ctypes.c_char_p, _dp, _dp, _dp]
    lib.ref_qr_shifts.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp,
                                  ctypes.POINTER(ctypes.c_int)]
    for f in ("ref_arnoldi_laplace",):
        getattr(lib, f).argtypes = [ctypes.c_int] * 3 + [_dp] * 3
    lib.ref_arnoldi_dense.argtypes = [ctypes.c_int] * 3 + [_dp] * 4
    lib.ref_laplace_apply.argtypes = [ctypes.c_int, _dp, _dp]
    lib.ref_bicgstabl_dense.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp,
                                        ctypes.POINTER(ctypes.c_int)]
    lib.ref_newton_cubic.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_double, _dp, _dp,
                                     ctypes.POINTER(ctypes.c_int), ctypes.c_double, ctypes.c_int]
    if a.linsolve_only:
        np.savez_compressed(os.path.join(a.out, "krylov_linsolve.npz"), **make_linsolve(lib))
        print("wrote krylov_linsolve.npz")
        return
    if not a.arnoldi_only:
        np.savez_compressed(os.path.join(a.out, "krylov_qr.npz"), **make_qr(lib))
        print("wrote krylov_qr.npz")
    if not a.host_only:
        np.savez_compressed(os.path.join(a.out, "krylov_arnoldi.npz"), **make_arnoldi(lib))
        print("wrote krylov_arnoldi.npz")


if __name__ == "__main__":
    main()
