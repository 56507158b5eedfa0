"""Python host mirror of the reference's Krylov eigen-analysis.

Follows Source/Arnoldi: ``Arnoldi_driver`` (Arnoldi_Driver.cu:29),
``select_shifts`` (Select_Shifts.cpp:86), ``QR_shifts`` (QR_Shifts.cpp:46)
and the restart loop of ``Implicit_restart_Arnoldi_GPU_data``
(Implicit_restart_Arnoldi.cu:444-581).  The Gram-Schmidt passes and the
restart run as sm_100a kernels behind the C ABI (include/ns3d.h); the small
m x m Hessenberg work stays on the host, as in the reference.

Storage follows the reference: the basis V is n x m column-major on the
device, held here as a contiguous float64 CUDA tensor of shape (m, n) (row j
is Krylov vector j, which is the same memory); H and Q are numpy (m, m)
matrices indexed [row, col].
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import (LaplaceContext, MAP_FN, MapContext, Ns3dError, ServedMapContext,
                   ShiftInvertContext, lib)

IM_EIG_TOL = 1.0e-15  # Source/Arnoldi/Macros.h:10


class _DeviceVector:
    """__cuda_array_interface__ view of a raw device pointer (no ownership)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8",
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": None}


class Map:
    """A matrix-vector map for :meth:`Krylov.arnoldi`: a C function pointer
    plus the context object it receives (kept alive here)."""

    def __init__(self, fn, ctx, keep=()):
        self.fn = fn
        self.ctx = ctx
        self._keep = keep

    @property
    def status(self) -> int:
        return int(self.ctx.status)

    def ctx_ptr(self) -> int:
        return ctypes.addressof(self.ctx)


class _ServedMap(Map):
    """A map whose context is an ns3d_served_map_context."""

    @property
    def status(self) -> int:
        return int(self.ctx.map.status)


class ShiftInvertMap(Map):
    """A shift-invert map (ns3d_shift_invert_context): the status lives in
    the embedded map context; the inner solves' counters are readable."""

    @property
    def status(self) -> int:
        return int(self.ctx.map.status)

    def stats(self) -> dict:
        c = self.ctx
        return {"last_flag": c.last_flag, "last_iter": c.last_iter, "last_tol": c.last_tol,
                "solves": c.solves, "inner_iter": c.inner_iter}


def select_shifts(H: np.ndarray, which: str = "LR"):
    """select_shifts (Select_Shifts.cpp:86-133): eigenvalues of H sorted by
    ``which`` ("LR" largest real part first, "LM" largest modulus first) and
    the Ritz estimates |last component| of the unit eigenvectors (zgeev)."""
    m = H.shape[0]
    w, vecs = np.linalg.eig(np.asarray(H, dtype=np.complex128))
    if which == "LR":
        key = -w.real
    elif which == "LM":
        key = -np.abs(w)
    else:
        raise ValueError("which must be 'LR' or 'LM'")
    order = np.argsort(key, kind="stable")
    return w[order], np.abs(vecs[m - 1, order])


def qr_shifts(k: int, H: np.ndarray, eigs):
    """QR_shifts through ns3d_qr_shifts (host code of the library).
    Returns (Q, H_new, ko)."""
    m = H.shape[0]
    L = lib()
    Q = np.zeros((m, m), order="F")
    Hf = np.asfortranarray(np.array(H, dtype=np.float64))
    e = np.asarray(eigs, dtype=np.complex128)
    er = np.ascontiguousarray(e.real)
    ei = np.ascontiguousarray(e.imag)
    ko = ctypes.c_int(0)
    rc = L.ns3d_qr_shifts(int(k), m, Q.ctypes.data, Hf.ctypes.data, er.ctypes.data,
                          ei.ctypes.data, ctypes.byref(ko))
    if rc != 0:
        raise Ns3dError(rc, "ns3d_qr_shifts")
    return np.ascontiguousarray(Q), np.ascontiguousarray(Hf), int(ko.value)


class Krylov:
    """One ns3d_krylov workspace: vectors of length n, bases of up to m_max
    columns, on one CUDA device."""

    def __init__(self, n: int, m_max: int, device=None):
        import torch

        self._torch = torch
        dev = torch.device(device if device is not None else "cuda")
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.n, self.m_max = int(n), int(m_max)
        self._L = lib()
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            torch.cuda.init()
            rc = self._L.ns3d_krylov_create(self.n, self.m_max, ctypes.byref(h))
        if rc != 0:
            raise Ns3dError(rc, "ns3d_krylov_create")
        self._h = h
        self._stream = None
        self._views = {}

    # -- plumbing ---------------------------------------------------------
    def _check(self, rc: int, where: str):
        if rc != 0:
            d = self._L.ns3d_krylov_last_error(self._h)
            raise Ns3dError(rc, where, d.decode() if d else "")

    def close(self):
        if getattr(self, "_h", None):
            self._L.ns3d_krylov_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream=None):
        """Run on a torch.cuda.Stream (None: the legacy default stream)."""
        self._stream = stream
        self._check(self._L.ns3d_krylov_set_stream(
            self._h, ctypes.c_void_p(stream.cuda_stream if stream is not None else 0)),
            "ns3d_krylov_set_stream")

    def _view(self, ptr: int):
        t = self._views.get(ptr)
        if t is None:
            t = self._torch.as_tensor(_DeviceVector(ptr, self.n), device=self.device)
            self._views[ptr] = t
        return t

    def python_map(self, fn) -> Map:
        """Wraps ``fn(x, y)`` (y = A x on float64 CUDA tensors of length n)."""
        torch = self._torch

        def tramp(_user, pin, pout):
            x, y = self._view(pin), self._view(pout)
            if self._stream is not None:
                with torch.cuda.stream(self._stream):
                    fn(x, y)
                self._stream.synchronize()
            else:
                fn(x, y)
                torch.cuda.current_stream(self.device).synchronize()

        cfn = MAP_FN(tramp)
        ctx = LaplaceContext()  # unused placeholder so every Map has a context
        return Map(cfn, ctx, keep=(tramp,))

    def laplace_map(self) -> Map:
        """The reference's Krylov self-test operator (ns3d_map_laplace1d)."""
        ctx = LaplaceContext(self.n, ctypes.c_void_p(
            self._stream.cuda_stream if self._stream is not None else 0), 0)
        return Map(ctypes.cast(self._L.ns3d_map_laplace1d, ctypes.c_void_p).value, ctx)

    def linearised_map(self, solver, U, Re: float, tau: float = 0.0) -> Map:
        """J(u) (minus 1/tau) on reduced vectors (ns3d_map_linearised)."""
        p = solver._fields(U, "U")
        ctx = MapContext(solver._h.value, p[0], p[1], p[2], 0, 0, 0, 0.0, float(Re),
                         float(tau), 0, 0)
        return Map(ctypes.cast(self._L.ns3d_map_linearised, ctypes.c_void_p).value, ctx,
                   keep=(U,))

    def exponential_map(self, solver, U, Vscratch, dt: float, Re: float, steps: int) -> Map:
        """``steps`` Heun tangent steps per call (ns3d_map_exponential); U
        advances with every call, as in the reference."""
        p = solver._fields(U, "U")
        q = solver._fields(Vscratch, "V")
        ctx = MapContext(solver._h.value, p[0], p[1], p[2], q[0], q[1], q[2], float(dt),
                         float(Re), 0.0, int(steps), 0)
        return Map(ctypes.cast(self._L.ns3d_map_exponential, ctypes.c_void_p).value, ctx,
                   keep=(U, Vscratch))

    def served_exponential_map(self, server, solver, U, Vscratch, dt: float, Re: float,
                               steps: int) -> Map:
        """What exponential_map computes, with every call's tangent steps run
        by ``server`` (a Server with a grid of solver's N) as a field request
        (ns3d_map_exponential_served): the Krylov driver's products share
        the device with the server's other requests.  The result's ``ctx``
        counts the requests served (``ctx.requests``)."""
        p = solver._fields(U, "U")
        q = solver._fields(Vscratch, "V")
        m = MapContext(solver._h.value, p[0], p[1], p[2], q[0], q[1], q[2], float(dt),
                       float(Re), 0.0, int(steps), 0)
        ctx = ServedMapContext(m, server._h.value, 0)
        return _ServedMap(ctypes.cast(self._L.ns3d_map_exponential_served,
                                      ctypes.c_void_p).value, ctx, keep=(U, Vscratch, server))

    def rhs_map(self, solver, U, Vscratch, Re: float) -> Map:
        """F(x) = RHS(unpack(x)) packed, writing unpack(x) into U first
        (ns3d_map_rhs, as NSCallRHS_reduced): a linearised_map on the same U
        is then the Jacobian at x."""
        p = solver._fields(U, "U")
        q = solver._fields(Vscratch, "V")
        ctx = MapContext(solver._h.value, p[0], p[1], p[2], q[0], q[1], q[2], 0.0, float(Re),
                         0.0, 0, 0)
        return Map(ctypes.cast(self._L.ns3d_map_rhs, ctypes.c_void_p).value, ctx,
                   keep=(U, Vscratch))

    def _shift_context(self, solver, U, Vscratch, dt, Re, steps, shift, angle, rotated,
                       L=6, tol=1e-9, max_iter=None, warm_start=False, inner=None):
        n = int(self._L.ns3d_krylov_length(solver._h))
        want = 2 * n if rotated else n
        p = solver._fields(U, "U")
        q = solver._fields(Vscratch, "V")
        m = MapContext(solver._h.value, p[0], p[1], p[2], q[0], q[1], q[2], float(dt), float(Re),
                       0.0, int(steps), 0)
        return want, ShiftInvertContext(
            m, float(shift), float(angle), int(L), float(tol),
            int(max_iter if max_iter is not None else n + 3), int(bool(warm_start)),
            inner._h.value if inner is not None else None, 0, 0, 0.0, 0, 0)

    def exponential_shifted_map(self, solver, U, Vscratch, dt: float, Re: float, steps: int,
                                shift: float, angle: float | None = None) -> ShiftInvertMap:
        """E - sigma (ns3d_map_exponential_shifted, NSCallMatrixVector_exponential_reduced)
        or, with ``angle``, its rotated real form on vectors of twice the
        length (ns3d_map_exponential_rotated); E = ``steps`` implicit tangent
        steps about the fixed base flow U.  This workspace's length must be
        the map's."""
        rotated = angle is not None
        want, ctx = self._shift_context(solver, U, Vscratch, dt, Re, steps, shift,
                                        angle or 0.0, rotated)
        if want != self.n:
            raise ValueError(f"the map acts on vectors of length {want}, this workspace on {self.n}")
        fn = self._L.ns3d_map_exponential_rotated if rotated else self._L.ns3d_map_exponential_shifted
        return ShiftInvertMap(ctypes.cast(fn, ctypes.c_void_p).value, ctx, keep=(U, Vscratch))

    def exponent_invert_map(self, solver, U, Vscratch, dt: float, Re: float, steps: int,
                            shift: float, angle: float | None = None, L: int = 6,
                            tol: float = 1.0e-9, max_iter: int | None = None,
                            warm_start: bool = False) -> ShiftInvertMap:
        """(E - sigma)^{-1} by BiCGStab(L) (ns3d_map_exponent_invert,
        Axb_exponent_invert) or, with ``angle``, (E - sigma e^{i angle})^{-1}
        in real form (ns3d_map_rotated_exponent_invert,
        Axb_rotated_exponent_invert).  The solves run in a workspace of their
        own; max_iter defaults to 3*Nx*Ny*Mz as in the reference
        (BiCG_Iter = N_Arnoldi, Source/NS3D_periodic.cu:1656)."""
        rotated = angle is not None
        n = int(self._L.ns3d_krylov_length(solver._h))
        want = 2 * n if rotated else n
        if want != self.n:
            raise ValueError(f"the map acts on vectors of length {want}, this workspace on {self.n}")
        inner = Krylov(want, 2, device=self.device)
        if self._stream is not None:
            inner.set_stream(self._stream)
        if max_iter is None:
            max_iter = n + 3
        _, ctx = self._shift_context(solver, U, Vscratch, dt, Re, steps, shift, angle or 0.0,
                                     rotated, L, tol, max_iter, warm_start, inner)
        fn = (self._L.ns3d_map_rotated_exponent_invert if rotated
              else self._L.ns3d_map_exponent_invert)
        return ShiftInvertMap(ctypes.cast(fn, ctypes.c_void_p).value, ctx,
                              keep=(U, Vscratch, inner))

    @staticmethod
    def _fnptr(A: Map) -> int:
        return A.fn if isinstance(A.fn, int) else ctypes.cast(A.fn, ctypes.c_void_p).value

    def bicgstabl(self, A: Map, x, rhs, L: int = 6, tol: float = 1e-9, maxiter: int = 1000):
        """BiCGStabL: solves A x = rhs in place (x: initial guess).  Returns
        (flag, iterations, relative residual) as the reference reports them."""
        self._vector(x)
        self._vector(rhs)
        t, it, fl = ctypes.c_double(tol), ctypes.c_int(maxiter), ctypes.c_int(0)
        self._check(self._L.ns3d_bicgstabl(self._h, int(L), ctypes.c_void_p(self._fnptr(A)),
                                           ctypes.c_void_p(A.ctx_ptr()),
                                           ctypes.c_void_p(x.data_ptr()),
                                           ctypes.c_void_p(rhs.data_ptr()), ctypes.byref(t),
                                           ctypes.byref(it), ctypes.byref(fl)), "ns3d_bicgstabl")
        return fl.value, it.value, t.value

    def newton(self, jacobian: Map, residual: Map, x, tol: float = 5e-7, maxiter: int = 1000,
               tol_linsolve: float = 1e-9, iter_linsolve: int = 1000) -> dict:
        """Newton: damped Newton iteration for residual(x) = 0, x in place."""
        self._vector(x)
        t, it = ctypes.c_double(tol), ctypes.c_int(maxiter)
        fl, lf = ctypes.c_int(0), ctypes.c_int(0)
        self._check(self._L.ns3d_newton(self._h, ctypes.c_void_p(self._fnptr(jacobian)),
                                        ctypes.c_void_p(jacobian.ctx_ptr()),
                                        ctypes.c_void_p(self._fnptr(residual)),
                                        ctypes.c_void_p(residual.ctx_ptr()),
                                        ctypes.c_void_p(x.data_ptr()), ctypes.byref(t),
                                        ctypes.byref(it), float(tol_linsolve), int(iter_linsolve),
                                        ctypes.byref(fl), ctypes.byref(lf)), "ns3d_newton")
        return {"flag": fl.value, "iterations": it.value, "tol": t.value,
                "linsolve_flag": lf.value}

    def _basis(self, V, m: int):
        torch = self._torch
        if (not isinstance(V, torch.Tensor) or V.dtype != torch.float64
                or V.device != self.device or V.dim() != 2 or V.shape[1] != self.n
                or V.shape[0] < m or not V.is_contiguous()):
            raise ValueError(f"V: expected a contiguous float64 ({m}, {self.n}) tensor on "
                             f"{self.device}")

    def _vector(self, f):
        torch = self._torch
        if (not isinstance(f, torch.Tensor) or f.dtype != torch.float64
                or f.device != self.device or f.numel() != self.n or not f.is_contiguous()):
            raise ValueError(f"f: expected a contiguous float64 vector of length {self.n}")

    # -- reference entry points ---------------------------------------------
    def arnoldi(self, A: Map, V, H: np.ndarray, f, k: int, m: int) -> dict:
        """Arnoldi_driver: extends the factorisation in place (V, f on the
        device, H host (m, m))."""
        self._basis(V, m)
        self._vector(f)
        Hf = np.asfortranarray(H[:m, :m], dtype=np.float64)
        fn = self._fnptr(A)
        rc = self._L.ns3d_arnoldi(self._h, ctypes.c_void_p(fn), ctypes.c_void_p(A.ctx_ptr()),
                                  ctypes.c_void_p(V.data_ptr()), Hf.ctypes.data,
                                  ctypes.c_void_p(f.data_ptr()), int(k), int(m))
        H[:m, :m] = Hf
        self._check(rc, "ns3d_arnoldi")
        mp, lh, nl = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int64(0)
        self._L.ns3d_krylov_stats(self._h, ctypes.byref(mp), ctypes.byref(lh), ctypes.byref(nl))
        return {"max_passes": mp.value, "limit_hits": lh.value, "launches": nl.value}

    def ira_restart(self, V, f, Q: np.ndarray, H: np.ndarray, k0: int) -> float:
        """Restart update f = hl V q + ql f, V = V Q; Q's columns k0.. are
        reset to the identity in place.  Returns ||f|| before the update."""
        m = Q.shape[0]
        self._basis(V, m)
        self._vector(f)
        Qf = np.asfortranarray(Q, dtype=np.float64)
        Hf = np.asfortranarray(H, dtype=np.float64)
        fn = ctypes.c_double(0.0)
        rc = self._L.ns3d_ira_restart(self._h, ctypes.c_void_p(V.data_ptr()),
                                      ctypes.c_void_p(f.data_ptr()), Qf.ctypes.data,
                                      Hf.ctypes.data, int(k0), m, ctypes.byref(fn))
        Q[:, :] = Qf
        self._check(rc, "ns3d_ira_restart")
        return fn.value

    def profile(self, V, ncols: int, x, reps: int = 10):
        """Per-launch device ms of the dot, update and restart kernels on
        ncols columns (see ns3d_krylov_profile)."""
        self._basis(V, ncols)
        self._vector(x)
        ms = (ctypes.c_double * 3)()
        self._check(self._L.ns3d_krylov_profile(self._h, ctypes.c_void_p(V.data_ptr()), ncols,
                                                ctypes.c_void_p(x.data_ptr()), reps, ms),
                    "ns3d_krylov_profile")
        return list(ms)

    def implicit_restart_arnoldi(self, A: Map, which: str = "LR", k: int = 6, m: int = 30,
                                 tol: float = 5.0e-8, max_iter: int = 3000, seed: int = 0,
                                 f0=None):
        """The restart loop of Implicit_restart_Arnoldi_GPU_data
        (Implicit_restart_Arnoldi.cu:531-581).  Returns (eigenvalues of H in
        'which' order, Ritz-norm, iterations, V, H).  The start vector is
        N(0, 2) from a seeded generator (the reference seeds from the clock)."""
        torch = self._torch
        if f0 is None:
            g = torch.Generator(device="cpu").manual_seed(int(seed))
            f = (torch.randn(self.n, generator=g, dtype=torch.float64) * 2.0).to(self.device)
        else:
            f = f0.clone()
        V = torch.zeros((m, self.n), dtype=torch.float64, device=self.device)
        H = np.zeros((m, m))
        k0, it, ritz_norm = 1, 0, 1.0
        eig = np.zeros(m, dtype=np.complex128)
        self.last_restart_columns = []  # Arnoldi columns built per cycle (map calls)
        self.last_restart_launches = 0  # kernels of the driver and the restarts (maps excluded)
        while it < max_iter and ritz_norm > tol:
            it += 1
            st = self.arnoldi(A, V, H, f, k0 - 1, m)
            self.last_restart_columns.append(m - k0 + 1)
            self.last_restart_launches += st["launches"] + 3  # + norm (2) and restart (1)
            eig, ritz = select_shifts(H, which)
            Q, H, k0 = qr_shifts(k, H, eig)
            if k0 < 1:
                raise Ns3dError(1, "implicit_restart_arnoldi", "no wanted Ritz value kept")
            fnorm = self.ira_restart(V, f, Q, H, k0)
            ritz[:k0] *= fnorm
            # vector_normC: max of fabsf (single precision), Products.cpp:23-31
            ritz_norm = float(np.max(np.abs(ritz[:k0]).astype(np.float32)))
        return eig, ritz_norm, it, V, H

    def implicit_restart_arnoldi_matrix_exponent(self, A_invert: Map, A: Map, which: str = "LR",
                                                 which_exponent: str = "LM", k: int = 6,
                                                 m: int = 30, tol: float = 5.0e-8,
                                                 max_iter: int = 3000, rotated: bool = False,
                                                 seed: int = 0, f0=None) -> dict:
        """Implicit_restart_Arnoldi_GPU_data_Matrix_Exponent
        (Implicit_restart_Arnoldi.cu:456-742): the restart loop on the
        shift-invert map ``A_invert`` with ``which_exponent`` ordering, on
        vectors of this workspace's length (twice the original length when
        ``rotated``), then the eigenpairs of the original map ``A`` from the
        converged Schur basis: :meth:`eigenpairs` (no rotation) or
        :meth:`eigenpairs_rotated`.  Returns a dict with the eigenvalues and
        eigenvectors of ``A`` sorted by ``which``, the residuals (real and
        imaginary parts for the rotated form), the Ritz norm, the
        iterations and the eigenvalues of the shift-invert map's H."""
        if rotated and self.n % 2:
            raise ValueError("a rotated workspace has even length")
        eig_h, ritz_norm, it, V, H = self.implicit_restart_arnoldi(
            A_invert, which_exponent, k, m, tol, max_iter, seed, f0)
        if A_invert.status != 0:
            raise Ns3dError(A_invert.status, "shift-invert map")
        if rotated:
            w, X, res_r, res_i = self.eigenpairs_rotated(A, V, H, k, which)
        else:
            w, X, res_r = self.eigenpairs(A, V, H, k, which)
            res_i = np.zeros_like(res_r)
        return {"eigenvalues": w, "eigenvectors": X, "residual_real": res_r,
                "residual_imag": res_i, "ritz_norm": ritz_norm, "iterations": it,
                "eigenvalues_invert": eig_h}

    # -- final stage of the implicit restart ----------------------------------
    def combine(self, V, C: np.ndarray, out=None):
        """W = V C on the device (ns3d_krylov_combine): V holds m basis
        vectors as rows of an (m, n) tensor, C is (m, p); returns the (p, n)
        tensor whose row j is sum_c C[c, j] V[c]."""
        torch = self._torch
        C = np.asfortranarray(C, dtype=np.float64)
        m, p = C.shape
        self._basis(V, m)
        W = out if out is not None else torch.empty((p, self.n), dtype=torch.float64,
                                                    device=self.device)
        self._basis(W, p)
        self._check(self._L.ns3d_krylov_combine(self._h, ctypes.c_void_p(V.data_ptr()), m,
                                                C.ctypes.data, p,
                                                ctypes.c_void_p(W.data_ptr())),
                    "ns3d_krylov_combine")
        return W

    def apply(self, A: Map, x, y):
        """y = A x through the map's C entry point (finished on return)."""
        fn = MAP_FN(self._fnptr(A)) if isinstance(A.fn, int) else A.fn
        fn(ctypes.c_void_p(A.ctx_ptr()), ctypes.c_void_p(x.data_ptr()),
           ctypes.c_void_p(y.data_ptr()))
        self._torch.cuda.synchronize(self.device)
        return y

    def eigenpairs(self, A: Map, V, H: np.ndarray, k: int, which: str = "LR"):
        """The final stage of Implicit_restart_Arnoldi_GPU_data
        (Implicit_restart_Arnoldi.cu:255-330, 589-664, no rotation): the real
        Schur form H_k = Z T Z^T of the leading k x k block (dhseqr there,
        scipy's LAPACK here), the Schur basis V1 = V_k Z, the Galerkin matrix
        R = V1^T A V1, its eigenpairs (R y = lambda y, unit y) sorted by
        ``which``, and the eigenvectors x = V1 y with the residuals
        ||A v1_i - V1 R e_i|| of the Schur vectors.  Returns (eigenvalues,
        eigenvectors as a complex (k, n) tensor, residuals).  The reference
        permutes the eigenvector columns a second time after sorting; here
        eigenvector i belongs to eigenvalue i."""
        from scipy.linalg import schur

        torch = self._torch
        _, Z = schur(np.asarray(H[:k, :k], dtype=np.float64), output="real")
        V1 = self.combine(V, Z)
        AV1 = torch.empty_like(V1)
        for i in range(k):
            self.apply(A, V1[i], AV1[i])
        R = (V1 @ AV1.T).cpu().numpy()               # R[i, j] = v1_i . A v1_j
        res = torch.linalg.vector_norm(AV1 - (torch.as_tensor(R, device=self.device).T @ V1),
                                       dim=1).cpu().numpy()
        w, Y = np.linalg.eig(R)
        key = -w.real if which == "LR" else -np.abs(w)
        order = np.argsort(key, kind="stable")
        w, Y = w[order], Y[:, order]
        X = torch.complex(self.combine(V1, Y.real), self.combine(V1, Y.imag))
        return w, X, res

    def eigenpairs_rotated(self, A: Map, V, H: np.ndarray, k: int, which: str = "LR"):
        """The rotated final stage, compute_eigensystem_of_original_mapping_rotation
        (Implicit_restart_Arnoldi.cu:335-434): the Schur basis V1 = V_k Z of
        the leading k x k block of H on this workspace's doubled vectors, its
        halves VR (real) and VI (imaginary), the Galerkin matrix
        R = VR^T A VR + VI^T A VI of the original map ``A`` (length n/2), the
        residuals ||A vr_i - VR R e_i|| and ||A vi_i - VI R e_i||, the
        eigenpairs of R sorted by ``which`` and the eigenvectors
        x = (VR + VI) y.  Returns (eigenvalues, eigenvectors as a complex
        (k, n/2) tensor, real residuals, imaginary residuals); eigenvector i
        belongs to eigenvalue i (the reference permutes the columns a second
        time after sorting)."""
        from scipy.linalg import schur

        torch = self._torch
        if self.n % 2:
            raise ValueError("a rotated workspace has even length")
        n2 = self.n // 2
        _, Z = schur(np.asarray(H[:k, :k], dtype=np.float64), output="real")
        V1 = self.combine(V, Z)
        VR, VI = V1[:, :n2].contiguous(), V1[:, n2:].contiguous()
        AVR, AVI = torch.empty_like(VR), torch.empty_like(VI)
        for i in range(k):
            self.apply(A, VR[i], AVR[i])
            self.apply(A, VI[i], AVI[i])
        R = (VR @ AVR.T + VI @ AVI.T).cpu().numpy()   # R[i, j] = vr_i . A vr_j + vi_i . A vi_j
        Rt = torch.as_tensor(R, device=self.device).T
        res_r = torch.linalg.vector_norm(AVR - Rt @ VR, dim=1).cpu().numpy()
        res_i = torch.linalg.vector_norm(AVI - Rt @ VI, dim=1).cpu().numpy()
        w, Y = np.linalg.eig(R)
        key = -w.real if which == "LR" else -np.abs(w)
        order = np.argsort(key, kind="stable")
        w, Y = w[order], Y[:, order]
        half = Krylov(n2, max(k, 2), device=self.device)
        try:
            VS = VR + VI
            X = torch.complex(half.combine(VS, Y.real), half.combine(VS, Y.imag))
        finally:
            half.close()
        return w, X, res_r, res_i
