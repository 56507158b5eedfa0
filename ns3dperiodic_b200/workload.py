"""Seeded synthetic inputs of the benchmark configurations (host, numpy).

Kolmogorov flow: body force f = (sin(n y), 0, 0) (unnormalised spectrum:
Im fx_hat(0, +-n, 0) = -+ Nx Ny Nz / 2), laminar profile
u0 = (Re/n^2) sin(n y) x, plus a seeded divergence-free perturbation with
Gaussian imaginary Fourier coefficients, amplitude spectrum |k|^-2 on
1 <= |k| <= 8, Hermitian on the kz = 0 / Nz/2 planes, Leray-projected with
the reference's projection entries (Source/math_support.cu:418-466) and
scaled to a relative L2 amplitude against u0.  Fields are complex128 arrays
(Nx, Ny, Nz//2+1) in the reference layout.
"""
from __future__ import annotations

import math

import numpy as np


def _signed(n):
    j = np.arange(n)
    return np.where(j >= n // 2, j - n, j)


def _leray(U, Nx, Ny, Nz, Lx, Ly, Lz):
    """u - AM.u with AM_ij = k_i k_j / |k|^2 (0 at k = 0)."""
    Mz = Nz // 2 + 1
    k1, k2, k3 = 2.0 * math.pi / Lx, 2.0 * math.pi / Ly, 2.0 * math.pi / Lz
    m = _signed(Nx)[:, None, None].astype(float)
    n = _signed(Ny)[None, :, None].astype(float)
    q = np.arange(Mz)[None, None, :].astype(float)
    din = k1 * k1 * m * m + k2 * k2 * n * n + k3 * k3 * q * q
    din = np.where(din == 0, 1.0, din)
    K = (k1 * m, k2 * n, k3 * q)
    kdotu = sum(K[i] * U[i] for i in range(3)) / din
    out = [U[i] - K[i] * kdotu for i in range(3)]
    for o in out:
        o[0, 0, 0] = 0
    return out


def kolmogorov_forcing(Nx, Ny, Nz, n=4):
    Mz = Nz // 2 + 1
    F = [np.zeros((Nx, Ny, Mz), np.complex128) for _ in range(3)]
    vol = float(Nx * Ny * Nz)
    F[0][0, n % Ny, 0] = -0.5j * vol
    F[0][0, (-n) % Ny, 0] = 0.5j * vol
    return F


def perturbation(Nx, Ny, Nz, seed, Lx=2 * math.pi, Ly=2 * math.pi, Lz=2 * math.pi,
                 kmin=1.0, kmax=8.0):
    """Unit-L2 (half spectrum) divergence-free odd perturbation."""
    Mz = Nz // 2 + 1
    rng = np.random.Generator(np.random.PCG64(seed))
    m = _signed(Nx)[:, None, None].astype(float)
    n = _signed(Ny)[None, :, None].astype(float)
    q = np.arange(Mz)[None, None, :].astype(float)
    kk = np.sqrt(m * m + n * n + q * q)
    amp = np.where((kk >= kmin) & (kk <= kmax), 1.0 / np.maximum(kk, 1.0) ** 2, 0.0)
    amp[Nx // 2, :, :] = 0.0
    amp[:, Ny // 2, :] = 0.0
    jm = (-np.arange(Nx)) % Nx
    km = (-np.arange(Ny)) % Ny
    U = []
    for _ in range(3):
        w = 1j * (rng.standard_normal((Nx, Ny, Mz)) * amp)
        for l in [0] + ([Nz // 2] if Nz % 2 == 0 and Nz // 2 < Mz else []):
            P = w[:, :, l].imag
            w[:, :, l] = 1j * (0.5 * (P - P[jm][:, km]))
        U.append(w)
    U = _leray(U, Nx, Ny, Nz, Lx, Ly, Lz)
    U = [1j * u.imag for u in U]
    for u in U:
        u[0, 0, 0] = 0.0
    nrm = math.sqrt(sum(float(np.vdot(u, u).real) for u in U))
    return [u / nrm for u in U]


def kolmogorov_state(N, Re, seed, rel_amp=1e-3, n=4):
    """(U, F) for the Kolmogorov workload on an N^3 2pi-periodic box."""
    F = kolmogorov_forcing(N, N, N, n)
    U0 = [F[0] * (Re / float(n * n)), np.zeros_like(F[0]), np.zeros_like(F[0])]
    P = perturbation(N, N, N, seed)
    base = math.sqrt(sum(float(np.vdot(u, u).real) for u in U0))
    return [U0[i] + rel_amp * base * P[i] for i in range(3)], F


def kolmogorov_dt(N, Re, cfl=0.3, n=4):
    """CFL time step from the laminar peak velocity Re/n^2: cfl * dx / max|u|."""
    return cfl * (2.0 * math.pi / N) / (Re / float(n * n))
