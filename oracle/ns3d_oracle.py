"""CPU oracle for the NS3DPeriodic pseudo-spectral path (TEST INFRASTRUCTURE).

This module is the checker, not the product.  Only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / reference legs of
``bench.py`` may import it.  The product path (``ns3dperiodic_b200``) never
routes through it.

It restates, in vectorised numpy/scipy FP64, the reference's algorithm for the
RK3 time step, the tangent (Jacobian-vector) steppers, the linearised RHS and
the Krylov packing, keeping every quirk of the reference:

* wave-number tables built with ``Mz`` passed as ``Nz`` and the x/y Nyquist
  index stored as ``-N/2`` (Source/math_support.cu:350-414,
  Source/NS3D_periodic.cu:1153-1161);
* the anisotropic "2/3" mask ``sqrt((m/Nx)^2+(n/Ny)^2+(q/Mz)^2) < 2/3`` with
  the (0,0,0) mode removed (Source/math_support.cu:471-519);
* the advective form ``Q_i = sum_j u_j d_j u_i`` built from 3 masked
  velocities and 9 masked gradients (Source/advection_2_3.cu:146-397,480-497);
* ``Re(Qhat) := 0`` everywhere and ``Qhat(0) := 0``
  (Source/advection_2_3.cu:35-70);
* the fused explicit-Euler update with the Leray matrix written as
  ``AM.Q - Q`` and unprojected forcing (Source/diffusion.cu:96-142);
* Shu-Osher SSP-RK3 (Source/RK_time_step.cu:310-327) and the Heun tangent
  stepper (Source/RK_time_step.cu:342-355).

Spectral fields use the reference layout: complex128 arrays of shape
``(Nx, Ny, Mz)`` with ``Mz = Nz//2 + 1`` (index macro ``IN(i,j,k)`` of
Source/Macros.h:11 with ``Nz = Mz``).  The forward transform is the
unnormalised real-to-complex 3-D DFT (cufftExecD2Z, Source/math_support.cu:301)
and the inverse is the complex-to-real DFT followed by ``1/(Nx Ny Nz)``
(Source/math_support.cu:325-334,123-150).  The complex-to-real transform uses
only the Hermitian part of the kz=0 and kz=Nz/2 planes (the imaginary part of
each z-line's DC and Nyquist bin is discarded after the x and y passes); this
is pocketfft's ``irfftn`` convention.

Parity status: pinned by the analytic Shapiro/laminar-Kolmogorov solutions
(tests/test_oracle_analytic.py) and by golden vectors produced with the
reference's own CUDA build (tests/golden/, made by tests/golden/make_golden.py
through oracle/_ref on a B200).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

try:  # scipy's pocketfft takes a thread count; numpy's does not
    import scipy.fft as _fft

    def _rfftn(a, workers):
        return _fft.rfftn(a, axes=(0, 1, 2), workers=workers)

    def _irfftn(a, shape, workers):
        return _fft.irfftn(a, s=shape, axes=(0, 1, 2), workers=workers)

except ImportError:  # pragma: no cover - scipy is in the image
    def _rfftn(a, workers):
        return np.fft.rfftn(a, axes=(0, 1, 2))

    def _irfftn(a, shape, workers):
        return np.fft.irfftn(a, s=shape, axes=(0, 1, 2))

PI = math.pi  # Source/Macros.h:74 (PI) and M_PI round to the same double


def _workers() -> int:
    return int(os.environ.get("NS3D_ORACLE_THREADS", os.cpu_count() or 1))


# ---------------------------------------------------------------------------
# Tables (host builders of the reference)
# ---------------------------------------------------------------------------

def _signed_index(n: int) -> np.ndarray:
    """m = j for j < n/2, j - n otherwise (Source/math_support.cu:354-357)."""
    j = np.arange(n)
    return np.where(j >= n // 2, j - n, j)


@dataclass
class Grid:
    """Reference wave-number, diffusion, Leray and mask tables.

    Built exactly as main() does: every builder receives ``Mz`` in its ``Nz``
    slot (Source/NS3D_periodic.cu:1153-1161).
    """

    Nx: int
    Ny: int
    Nz: int
    Lx: float = 2.0 * PI
    Ly: float = 2.0 * PI
    Lz: float = 2.0 * PI
    Mz: int = field(init=False)

    def __post_init__(self):
        self.Mz = self.Nz // 2 + 1
        Nx, Ny, Mz = self.Nx, self.Ny, self.Mz
        m = _signed_index(Nx)
        n = _signed_index(Ny)
        q = np.arange(Mz)  # no wrap in z: "due to reality condition"
        self.m, self.n, self.q = m, n, q
        # build_Nabla_Wavenumbers / build_Laplace_Wavenumbers (math_support.cu:350-414)
        self.kx = 2.0 * PI / self.Lx * m
        self.ky = 2.0 * PI / self.Ly * n
        self.kz = 2.0 * PI / self.Lz * q
        KX = self.kx[:, None, None]
        KY = self.ky[None, :, None]
        KZ = self.kz[None, None, :]
        # build_Laplace_and_Diffusion (math_support.cu:374-390): din_diffusion = |k|^2
        self.din_diffusion = KX * KX + KY * KY + KZ * KZ
        # build_projection_matrix_elements (math_support.cu:418-466)
        k1 = 2.0 * PI / self.Lx
        k2 = 2.0 * PI / self.Ly
        k3 = 2.0 * PI / self.Lz
        M = m[:, None, None].astype(np.float64)
        Nn = n[None, :, None].astype(np.float64)
        Q = q[None, None, :].astype(np.float64)
        din = k1 * k1 * M * M + k2 * k2 * Nn * Nn + k3 * k3 * Q * Q
        zero = (m[:, None, None] ** 2 + n[None, :, None] ** 2 + q[None, None, :] ** 2) == 0
        din = np.where(zero, 1.0, din)
        self.AM11 = k1 * k1 * M * M / din
        self.AM22 = k2 * k2 * Nn * Nn / din
        self.AM33 = k3 * k3 * Q * Q / din
        self.AM12 = k1 * k2 * M * Nn / din
        self.AM13 = k1 * k3 * M * Q / din
        self.AM23 = k2 * k3 * Nn * Q / din
        for a in (self.AM11, self.AM22, self.AM33, self.AM12, self.AM13, self.AM23):
            a[0, 0, 0] = 0.0
        # build_mask_matrix (math_support.cu:471-519), called with Nz=Mz
        kxs = m[:, None, None] * 2 * PI / self.Lx
        kys = n[None, :, None] * 2 * PI / self.Ly
        kzs = q[None, None, :] * 2 * PI / self.Lz
        kxMax = 2 * Nx * PI / self.Lx
        kyMax = 2 * Ny * PI / self.Ly
        kzMax = 2 * Mz * PI / self.Lz
        sphere2 = np.sqrt(kxs * kxs / (kxMax * kxMax) + kys * kys / (kyMax * kyMax)
                          + kzs * kzs / (kzMax * kzMax))
        mask = np.where(sphere2 < 2.0 / 3.0, 1.0, 0.0)
        self.mask_sphere = mask.copy()  # before the (0,0,0) removal
        mask[0, 0, 0] = 0.0
        self.mask = mask

    @property
    def shape_c(self):
        return (self.Nx, self.Ny, self.Mz)

    @property
    def shape_r(self):
        return (self.Nx, self.Ny, self.Nz)

    @property
    def dx(self):
        return self.Lx / self.Nx

    @property
    def dy(self):
        return self.Ly / self.Ny

    @property
    def dz(self):
        return self.Lz / self.Nz

    def mask_cutoff(self) -> np.ndarray:
        """Per (x, y) column the number of leading kz modes the mask keeps.

        The mask is monotone in q for every (j, k); this checks it and returns
        ``qcut[j, k]`` so that mask(j,k,l) = (l < qcut[j,k]) except (0,0,0).
        """
        m = self.mask_sphere
        qcut = m.sum(axis=2).astype(np.int32)
        l = np.arange(self.Mz)[None, None, :]
        if not np.array_equal(m, (l < qcut[:, :, None]).astype(np.float64)):
            raise AssertionError("dealiasing mask is not a kz-prefix")
        return qcut


# ---------------------------------------------------------------------------
# Transforms
# ---------------------------------------------------------------------------

def c2r(g: Grid, X: np.ndarray) -> np.ndarray:
    """iFFTN_Device: Z2D then *1/(Nx Ny Nz) (Source/math_support.cu:325-334)."""
    return _irfftn(X, g.shape_r, _workers())


def r2c(g: Grid, x: np.ndarray) -> np.ndarray:
    """FFTN_Device: unnormalised D2Z (Source/math_support.cu:301-312)."""
    return _rfftn(x, _workers())


def _ik(U: np.ndarray, k: np.ndarray) -> np.ndarray:
    """build_ders_device: der.x = -U.y*k, der.y = U.x*k (advection_2_3.cu:206-213)."""
    return (-U.imag * k) + 1j * (U.real * k)


def _set_to_zero_real(Q):
    """set_to_zero_real (Source/advection_2_3.cu:35-70)."""
    for q in Q:
        q.real[...] = 0.0
        q[0, 0, 0] = 0.0
    return Q


def _physical_fields(g: Grid, U):
    """Masked velocities and masked gradients in physical space.

    build_vels_and_ders + filter_wavenumbers + the C2R calls of convolute_2p3
    (Source/advection_2_3.cu:320-330,348-355,359-389).  Returns (u, du) with
    du[i][j] = d_j u_i.
    """
    KX = g.kx[:, None, None]
    KY = g.ky[None, :, None]
    KZ = g.kz[None, None, :]
    u = [c2r(g, Ui * g.mask) for Ui in U]
    du = []
    for Ui in U:
        du.append([c2r(g, _ik(Ui, KX) * g.mask),
                   c2r(g, _ik(Ui, KY) * g.mask),
                   c2r(g, _ik(Ui, KZ) * g.mask)])
    return u, du


def convolution(g: Grid, U):
    """calculate_convolution_2p3 (Source/advection_2_3.cu:480-497).

    Qhat_i = FFT[ sum_j (M u_j)(d_j M u_i) ], then Re(Qhat)=0, Qhat(0)=0.
    """
    u, du = _physical_fields(g, U)
    Q = []
    for i in range(3):
        # calc_vels_nabla_vels: ux*der_x + uy*der_y + uz*der_z (advection_2_3.cu:245)
        q = u[0] * du[i][0] + u[1] * du[i][1] + u[2] * du[i][2]
        Q.append(r2c(g, q))
    return _set_to_zero_real(Q)


def convolution_uv(g: Grid, U, V):
    """calculate_convolution_2p3_UV (Source/advection_2_3.cu:500-525).

    Qhat_i = FFT[ (v.grad) u_i + (u.grad) v_i ] on masked fields
    (convolute_2p3_UV, Source/advection_2_3.cu:401-475).
    """
    u, du = _physical_fields(g, U)
    v, dv = _physical_fields(g, V)
    Q = []
    for i in range(3):
        q = v[0] * du[i][0] + v[1] * du[i][1] + v[2] * du[i][2]
        q = q + (u[0] * dv[i][0] + u[1] * dv[i][1] + u[2] * dv[i][2])
        Q.append(r2c(g, q))
    return _set_to_zero_real(Q)


def _am_q(g: Grid, Q):
    """AM.Q with the 6 stored Leray entries (Source/diffusion.cu:116-123)."""
    Qx, Qy, Qz = Q
    return (g.AM11 * Qx + g.AM12 * Qy + g.AM13 * Qz,
            g.AM12 * Qx + g.AM22 * Qy + g.AM23 * Qz,
            g.AM13 * Qx + g.AM23 * Qy + g.AM33 * Qz)


# ---------------------------------------------------------------------------
# Pointwise spectral updates (Source/diffusion.cu)
# ---------------------------------------------------------------------------

def update_explicit(g: Grid, U, F, Q, dt, Re):
    """solve_advection_diffusion_projection_device (diffusion.cu:96-142)."""
    AMQ = _am_q(g, Q)
    G = 1.0 - g.din_diffusion * dt / Re
    return [dt * AMQ[i] + G * U[i] + dt * F[i] - dt * Q[i] for i in range(3)]


def update_explicit_uv(g: Grid, V, Q, dt, Re):
    """solve_advection_diffusion_projection_device_UV (diffusion.cu:209-259)."""
    AMQ = _am_q(g, Q)
    G = 1.0 - g.din_diffusion * dt / Re
    return [dt * AMQ[i] + G * V[i] - dt * Q[i] for i in range(3)]


def update_uv_rhs(g: Grid, V, Q, Re):
    """solve_advection_diffusion_projection_device_UV_RHS (diffusion.cu:144-206)."""
    AMQ = _am_q(g, Q)
    G = -g.din_diffusion / Re
    return [AMQ[i] + G * V[i] - Q[i] for i in range(3)]


def update_implicit_uv(g: Grid, V, Q, dt, Re):
    """solve_advection_implicit_diffusion_projection_device_UV (diffusion.cu:264-314)."""
    AMQ = _am_q(g, Q)
    G = 1.0 + g.din_diffusion * dt / Re
    return [(dt * AMQ[i] + V[i] - dt * Q[i]) / G for i in range(3)]


def rhs_update(g: Grid, U, F, Q, Re):
    """RHS_advection_diffusion_projection_device (diffusion.cu:319-365)."""
    AMQ = _am_q(g, Q)
    G = -g.din_diffusion / Re
    return [AMQ[i] + G * U[i] + F[i] - Q[i] for i in range(3)]


# ---------------------------------------------------------------------------
# Steppers (Source/RK_time_step.cu)
# ---------------------------------------------------------------------------

def single_time_step(g: Grid, U, F, dt, Re):
    """single_time_step (RK_time_step.cu:248-263): u <- u + dt*L(u)."""
    return update_explicit(g, U, F, convolution(g, U), dt, Re)


def rk3_ssp(g: Grid, U, F, dt, Re):
    """RK3_SSP (RK_time_step.cu:310-327), returns the new state."""
    U1 = [u.copy() for u in U]
    U1 = single_time_step(g, U1, F, dt, Re)
    U1 = single_time_step(g, U1, F, dt, Re)
    U2 = [3.0 / 4.0 * U[i] + 1.0 / 4.0 * U1[i] for i in range(3)]
    U2 = single_time_step(g, U2, F, dt, Re)
    return [1.0 / 3.0 * U[i] + 2.0 / 3.0 * U2[i] for i in range(3)]


def return_rhs(g: Grid, U, F, Re):
    """return_RHS (RK_time_step.cu:231-245)."""
    return rhs_update(g, U, F, convolution(g, U), Re)


def single_time_step_uv(g: Grid, U, V, dt, Re):
    """single_time_step_UV (RK_time_step.cu:265-278): v <- v + dt*J(u)v."""
    return update_explicit_uv(g, V, convolution_uv(g, U, V), dt, Re)


def rk3_ssp_uv_rhs(g: Grid, U, V, dt, Re):
    """RK3_SSP_UV_RHS (RK_time_step.cu:330-338): v <- J(u) v."""
    return update_uv_rhs(g, V, convolution_uv(g, U, V), Re)


def single_time_step_iuv_rhs(g: Grid, U, V, dt, Re):
    """single_time_step_iUV_RHS (RK_time_step.cu:296-306)."""
    return update_implicit_uv(g, V, convolution_uv(g, U, V), dt, Re)


def rk3_ssp_uv(g: Grid, U, V, F, dt, Re):
    """RK3_SSP_UV (RK_time_step.cu:342-355): Heun tangent with RK3 base.

    Returns (U_new, V_new); the reference advances the base state in place.
    """
    V1 = single_time_step_uv(g, U, V, dt, Re)
    Un = rk3_ssp(g, U, F, dt, Re)
    V1 = single_time_step_uv(g, Un, V1, dt, Re)
    return Un, [0.5 * V[i] + 0.5 * V1[i] for i in range(3)]


# ---------------------------------------------------------------------------
# Krylov vector packing (Source/NS3D_periodic.cu:173-317)
# ---------------------------------------------------------------------------

def pack_reduced(V) -> np.ndarray:
    """A_vector_from_velocities_reduced_kernel: Im parts, mode 0 dropped."""
    return np.concatenate([v.reshape(-1)[1:].imag for v in V])


def unpack_reduced(g: Grid, vec: np.ndarray):
    """velocities_from_A_vector_reduced_kernel: Re := 0, mode 0 := 0."""
    nc = g.Nx * g.Ny * g.Mz
    out = []
    for c in range(3):
        f = np.zeros(nc, dtype=np.complex128)
        f[1:] = 1j * vec[c * (nc - 1):(c + 1) * (nc - 1)]
        out.append(f.reshape(g.shape_c))
    return out


def linearised_matvec_reduced(g: Grid, U, vec, dt, Re):
    """NSCallMatrixVector_reduced (NS3D_periodic.cu:340-361): J(u)v on packed vectors."""
    V = unpack_reduced(g, vec)
    return pack_reduced(rk3_ssp_uv_rhs(g, U, V, dt, Re))


def exponential_shifted_reduced(g: Grid, U, vec, dt, Re, steps: int, shift: float):
    """NSCallMatrixVector_exponential_reduced (NS3D_periodic.cu:473-500):
    ``steps`` single_time_step_iUV_RHS of v = unpack(vec) about the fixed U,
    then A_vector_from_velocities_reduced_shifted_kernel (NS3D_periodic.cu:
    253-270): Im v(1..) - shift * vec."""
    V = unpack_reduced(g, vec)
    for _ in range(steps):
        V = single_time_step_iuv_rhs(g, U, V, dt, Re)
    return pack_reduced(V) - shift * vec


def exponential_rotated_reduced(g: Grid, U, vec, dt, Re, steps: int, shift: float,
                                angle: float):
    """NSCallMatrixVector_exponential_rotated_reduced (NS3D_periodic.cu:
    552-586) on a doubled vector [real half; imaginary half]:
    out_r = E in_r - sr in_r + si in_i and out_i = E in_i - sr in_i - si in_r
    with (sr, si) = shift (cos angle, sin angle)
    (A_vector_from_velocities_reduced_shifted_rotated_kernel_Real/_Imag,
    NS3D_periodic.cu:273-300)."""
    n = vec.size // 2
    sr, si = shift * math.cos(angle), shift * math.sin(angle)
    xr, xi = vec[:n], vec[n:]

    def e(x):
        V = unpack_reduced(g, x)
        for _ in range(steps):
            V = single_time_step_iuv_rhs(g, U, V, dt, Re)
        return pack_reduced(V)

    return np.concatenate([e(xr) - sr * xr + si * xi, e(xi) - sr * xi - si * xr])


# ---------------------------------------------------------------------------
# Diagnostics (Source/math_support.cu:720-806, divergence.cu:8-31)
# ---------------------------------------------------------------------------

def physical_velocity(g: Grid, U):
    return [c2r(g, u) for u in U]


def kinetic_energy(g: Grid, U) -> float:
    """get_kinetic_energy: sum 0.5*(uy^2+uz^2)*dx*dy (transverse energy only)."""
    _, uy, uz = physical_velocity(g, U)
    return float(np.sum(0.5 * (uy * uy + uz * uz) * g.dx * g.dy))


def dissipation(g: Grid, U) -> float:
    """get_dissipation: FD central differences without the 1/2 (math_support.cu:755-797)."""
    ux, uy, uz = physical_velocity(g, U)

    def d(a, ax, h):
        return (np.roll(a, -1, axis=ax) - np.roll(a, 1, axis=ax)) / h

    dx, dy, dz = g.dx, g.dy, g.dz
    uxx, uxy, uxz = d(ux, 0, dx), d(ux, 1, dy), d(ux, 2, dz)
    uyx, uyy, uyz = d(uy, 0, dx), d(uy, 1, dy), d(uy, 2, dz)
    uzx, uzy, uzz = d(uz, 0, dx), d(uz, 1, dy), d(uz, 2, dz)
    dens = dx * dy * dz * (2.0 * (uxx * uxx + uyy * uyy + uzz * uzz)
                           + (uyz + uzy) ** 2 + (uxz + uzx) ** 2 + (uxy + uyx) ** 2)
    return float(np.sum(dens))


def divergence_hat(g: Grid, U, dt=1.0):
    """solve_divergence: div_hat = i k.u / dt (divergence.cu:8-31)."""
    KX = g.kx[:, None, None]
    KY = g.ky[None, :, None]
    KZ = g.kz[None, None, :]
    re = (-U[0].imag * KX - U[1].imag * KY - U[2].imag * KZ) / dt
    im = (U[0].real * KX + U[1].real * KY + U[2].real * KZ) / dt
    return re + 1j * im


# ---------------------------------------------------------------------------
# Inputs: analytic fields and the seeded Kolmogorov workload
# ---------------------------------------------------------------------------

def shapiro_physical(g: Grid, t: float, Re: float):
    """Shapiro's Beltrami field (NS3D_periodic.cu:810-829, Shapiro_test.cu:24-31)."""
    x = (np.arange(g.Nx) * g.dx)[:, None, None]
    y = (np.arange(g.Ny) * g.dy)[None, :, None]
    z = (np.arange(g.Nz) * g.dz)[None, None, :]
    factor = math.sqrt(3.0)
    e = math.exp(-(factor * factor) * t / Re)
    ux = -0.5 * (factor * np.cos(x) * np.sin(y) * np.sin(z) + np.sin(x) * np.cos(y) * np.cos(z)) * e
    uy = 0.5 * (factor * np.sin(x) * np.cos(y) * np.sin(z) - np.cos(x) * np.sin(y) * np.cos(z)) * e
    uz = np.cos(x) * np.cos(y) * np.sin(z) * e
    shape = g.shape_r
    return [np.broadcast_to(a, shape).copy() for a in (ux, uy, uz)]


def shapiro_hat(g: Grid, t: float, Re: float):
    return [r2c(g, a) for a in shapiro_physical(g, t, Re)]


def kolmogorov_forcing(g: Grid, n: int = 4):
    """f = (sin(n y), 0, 0): Im fx_hat(0, +-n, 0) = -+ Nx Ny Nz / 2."""
    F = [np.zeros(g.shape_c, dtype=np.complex128) for _ in range(3)]
    vol = float(g.Nx * g.Ny * g.Nz)
    F[0][0, n % g.Ny, 0] = -0.5j * vol
    F[0][0, (-n) % g.Ny, 0] = 0.5j * vol
    return F


def leray_project(g: Grid, U):
    """u - AM.u with the reference's Leray entries."""
    AMU = _am_q(g, U)
    return [U[i] - AMU[i] for i in range(3)]


def _hermitian_odd_planes(g: Grid, W: np.ndarray) -> np.ndarray:
    """Make a pure-imaginary half spectrum Hermitian on the kz=0 and kz=Nz/2 planes."""
    W = W.copy()
    jm = (-np.arange(g.Nx)) % g.Nx
    km = (-np.arange(g.Ny)) % g.Ny
    planes = [0] + ([g.Nz // 2] if g.Nz % 2 == 0 and g.Nz // 2 < g.Mz else [])
    for l in planes:
        P = W[:, :, l].imag
        P = 0.5 * (P - P[jm][:, km])  # Im(-k) = -Im(k)
        W[:, :, l] = 1j * P
    return W


def random_perturbation(g: Grid, seed: int, kmin: float = 1.0, kmax: float = 8.0):
    """Seeded divergence-free perturbation: Gaussian Im parts, |k|^-2 amplitude.

    Pure imaginary (odd fields), Hermitian on the kz=0 / kz=Nz/2 planes, zero
    mean, zero on the x/y Nyquist lines, Leray-projected.  Unit L2 norm over
    the half spectrum.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    m = g.m[:, None, None].astype(np.float64)
    n = g.n[None, :, None].astype(np.float64)
    q = g.q[None, None, :].astype(np.float64)
    kk = np.sqrt(m * m + n * n + q * q)
    amp = np.where((kk >= kmin) & (kk <= kmax), 1.0 / np.maximum(kk, 1.0) ** 2, 0.0)
    amp[g.Nx // 2, :, :] = 0.0
    amp[:, g.Ny // 2, :] = 0.0
    U = []
    for _ in range(3):
        w = rng.standard_normal(g.shape_c) * amp
        U.append(_hermitian_odd_planes(g, 1j * w))
    U = leray_project(g, U)
    U = [1j * u.imag for u in U]
    for u in U:
        u[0, 0, 0] = 0.0
    nrm = math.sqrt(sum(float(np.vdot(u, u).real) for u in U))
    return [u / nrm for u in U]


def kolmogorov_state(g: Grid, Re: float, seed: int, rel_amp: float = 1e-3, n: int = 4):
    """Laminar Kolmogorov profile (Re/n^2) sin(n y) x plus a seeded perturbation."""
    F = kolmogorov_forcing(g, n)
    U0 = [F[0] * (Re / float(n * n)), np.zeros(g.shape_c, np.complex128),
          np.zeros(g.shape_c, np.complex128)]
    P = random_perturbation(g, seed)
    base = math.sqrt(sum(float(np.vdot(u, u).real) for u in U0))
    U = [U0[i] + rel_amp * base * P[i] for i in range(3)]
    return U, F


def cfl_dt(g: Grid, U, cfl: float = 0.3) -> float:
    """dt = cfl * min(dx) / max|u| evaluated on the physical field."""
    u = physical_velocity(g, U)
    umax = float(np.max(np.sqrt(u[0] ** 2 + u[1] ** 2 + u[2] ** 2)))
    return cfl * min(g.dx, g.dy, g.dz) / umax


def rel_l2(A, B) -> float:
    num = sum(float(np.vdot(A[i] - B[i], A[i] - B[i]).real) for i in range(len(A)))
    den = sum(float(np.vdot(B[i], B[i]).real) for i in range(len(B)))
    return math.sqrt(num / den) if den > 0 else math.sqrt(num)


# ---------------------------------------------------------------------------
# Filters, curl, the per-step diagnostic record and the energy spectrum
# (Source/math_support.cu:680-717,819-987; Source/NS3D_periodic.cu:1291-1452,
# 1853; Source/Shapiro_test.cu:8-50)
# ---------------------------------------------------------------------------

def helmholtz_filter(g: Grid, U, eps: float):
    """Helmholz_Fourier_Filter_Device (math_support.cu:866-907): u/(1+eps^2|k|^2),
    signed x/y indices (Nyquist -> -N/2), z index as stored."""
    KX = (2.0 * PI / g.Lx * g.m)[:, None, None]
    KY = (2.0 * PI / g.Ly * g.n)[None, :, None]
    KZ = (2.0 * PI / g.Lz * g.q)[None, None, :]
    filt = 1.0 / (1.0 + eps * eps * (KX * KX + KY * KY + KZ * KZ))
    return [filt * u for u in U]


def cutoff_mask(g: Grid, radius: float) -> np.ndarray:
    """CutOff_Fourier_Filter_Device (math_support.cu:929-970), launched with Mz
    in its Nz slot: keep m^2/Nx^2 + n^2/Ny^2 + q^2/Mz^2 <= radius^2."""
    m = g.m[:, None, None].astype(np.float64)
    n = g.n[None, :, None].astype(np.float64)
    q = g.q[None, None, :].astype(np.float64)
    r2 = (1.0 * m * m / (1.0 * g.Nx * g.Nx) + 1.0 * n * n / (1.0 * g.Ny * g.Ny)
          + 1.0 * q * q / (1.0 * g.Mz * g.Mz))
    return (r2 <= radius * radius).astype(np.float64)


def cutoff_filter(g: Grid, U, radius: float):
    mask = cutoff_mask(g, radius)
    return [mask * u for u in U]


def curl_fd(g: Grid, u):
    """get_curl_device (math_support.cu:680-707) on physical fields: central
    differences with periodic wrap, including the reference's rot_y term
    0.5 (uz(j+1) - ux(j-1)) / dx (it mixes uz and ux)."""
    ux, uy, uz = u

    def sh(a, ax, s):  # a(index + s) with periodic wrap
        return np.roll(a, -s, axis=ax)

    dx, dy, dz = g.dx, g.dy, g.dz
    rx = 0.5 * (sh(uz, 1, 1) - sh(uz, 1, -1)) / dy - 0.5 * (sh(uy, 2, 1) - sh(uy, 2, -1)) / dz
    ry = 0.5 * (sh(ux, 2, 1) - sh(ux, 2, -1)) / dz - 0.5 * (sh(uz, 0, 1) - sh(ux, 0, -1)) / dx
    rz = 0.5 * (sh(uy, 0, 1) - sh(uy, 0, -1)) / dx - 0.5 * (sh(ux, 1, 1) - sh(ux, 1, -1)) / dy
    return [rx, ry, rz]


def _flat_r(g: Grid, i, j, k) -> int:
    """IN(i,j,k) of a physical field (Macros.h:11), as a flat index."""
    return i * (g.Ny * g.Nz) + j * g.Nz + k


def _flat_c(g: Grid, i, j, k) -> int:
    """IN(i,j,k) with Nz = Mz: a spectral field's flat index."""
    return i * (g.Ny * g.Mz) + j * g.Mz + k


def record_points(g: Grid):
    """Flat indices the time loop reads (NS3D_periodic.cu:1357-1450): three
    physical probes and eleven spectral ones."""
    Nx, Ny, Nz, Mz = g.Nx, g.Ny, g.Nz, g.Mz
    phys = [_flat_r(g, Nx // 2 - 4, Ny // 2 - 3, Nz // 2 - 2),
            _flat_r(g, Nx // 3, Ny // 3, Nz // 3),
            _flat_r(g, Nx // 8, Ny // 8, Nz // 8)]
    spec = [_flat_c(g, Nx - 6, Ny - 6, Mz - 6),
            _flat_c(g, Nx // 5, Ny // 4 - 3, Mz // 4 - 1),
            _flat_c(g, Nx // 5, Ny // 5, Mz // 5),
            _flat_c(g, 2, 2, 2), _flat_c(g, 1, 0, 0), _flat_c(g, 0, 0, 0),
            _flat_c(g, 1, 1, 0), _flat_c(g, 1, 1, 1), _flat_c(g, Nx - 1, 0, 0),
            _flat_c(g, Nx - 1, Ny - 1, 0), _flat_c(g, Nx - 1, Ny - 1, Mz - 1)]
    return phys, spec


def series_record(g: Grid, U, total_time: float, Re: float) -> np.ndarray:
    """The 50 columns the time loop writes to time_dependant.dat per step
    (NS3D_periodic.cu:1324-1452), computed the reference's way: physical
    velocity (Image_to_Domain), the cut-off filtered velocity (the Helmholtz
    filter's output is overwritten by CutOff_Fourier_Filter with radius 0.1),
    finite-difference curls, get_kinetic_energy / get_dissipation, point
    reads by flat index, and Re/Im reads of the spectral state."""
    phys, spec = record_points(g)
    u = physical_velocity(g, U)
    r = curl_fd(g, u)
    uf = physical_velocity(g, cutoff_filter(g, U, 0.1))
    rf = curl_fd(g, uf)
    e = kinetic_energy(g, U)
    d = dissipation(g, U)
    flat = lambda a, i: float(a.reshape(-1)[i])  # noqa: E731
    Ur = [x.reshape(-1) for x in U]
    col = [total_time]
    for p, tail in zip(phys, (e, d, e - d / Re)):
        col += [flat(a, p) for a in u] + [flat(a, p) for a in r] + [tail]
    p = phys[1]
    col += [flat(a, p) for a in uf] + [flat(a, p) for a in rf] + [e]
    s = spec[0]
    col += [Ur[0][s].real, Ur[0][s].imag, Ur[1][s].real, Ur[1][s].imag,
            Ur[2][s].real, Ur[2][s].imag, d]
    a, b = spec[1], spec[2]
    col += [Ur[0][a].imag, Ur[0][b].imag, Ur[1][a].imag, Ur[1][b].imag,
            Ur[2][a].imag, Ur[2][b].imag, Ur[0][spec[3]].imag]
    col += [Ur[0][i].imag for i in spec[4:]]
    return np.array(col, dtype=np.float64)


def format_series_line(rec) -> str:
    """One time_dependant.dat line: 50 '%le' fields, single spaces."""
    return " ".join("%e" % v for v in rec) + "\n"


def energy_spectrum(g: Grid, U) -> np.ndarray:
    """calculate_energy_spectrum (math_support.cu:819-860): bins n = j+k+l over
    j < Nx/2, k < Ny/2, l < Mz; E[n] = sum |u_hat|^2 / norm^2 with norm =
    Nx*Ny*Mz (the function receives Mz as Nz).  Returns the unhalved sums."""
    Nx, Ny, Mz = g.Nx, g.Ny, g.Mz
    size = Nx // 2 + Ny // 2 + Mz
    norm = float(Nx * Ny * Mz)
    E = np.zeros(size)
    j = np.arange(Nx // 2)[:, None, None]
    k = np.arange(Ny // 2)[None, :, None]
    l = np.arange(Mz)[None, None, :]
    n = np.broadcast_to(j + k + l, (Nx // 2, Ny // 2, Mz)).reshape(-1)
    dens = sum((u[: Nx // 2, : Ny // 2, :].real ** 2 / norm / norm
                + u[: Nx // 2, : Ny // 2, :].imag ** 2 / norm / norm) for u in U).reshape(-1)
    np.add.at(E, n, dens)
    return E


def format_energy_spectrum(g: Grid, E) -> str:
    """Ek.dat text: '%i %.16le %.16le' per bin; bins no mode reaches print 0."""
    size = len(E)
    nmax = (g.Nx // 2 - 1) + (g.Ny // 2 - 1) + (g.Mz - 1)
    out = []
    with np.errstate(divide="ignore"):
        for n in range(size):
            if n <= nmax:
                out.append("%i %.16e %.16e\n" % (n, 0.5 * E[n], 0.5 * (0.5 * math.pow(n, -5.0 / 3.0)
                                                                       if n else math.inf)))
            else:
                out.append("%i %.16e %.16e\n" % (0, 0.0, 0.0))
    return "".join(out)


def shapiro_error(g: Grid, U, t: float, Re: float) -> float:
    """Shapiro_test_case (Shapiro_test.cu:8-50): max over the grid of
    |u - u_exact(t)| (Euclidean norm per point) on the physical field."""
    u = physical_velocity(g, U)
    ex = shapiro_physical(g, t, Re)
    err = np.sqrt(sum((a - b) ** 2 for a, b in zip(u, ex)))
    return float(np.max(err))
