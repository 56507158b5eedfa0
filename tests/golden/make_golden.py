"""Generate golden vectors from the reference's own CUDA build.

Runs the unmodified reference path (oracle/_ref/libns3d_ref.so, built by
oracle/Makefile from the reference sources) on a GPU, on small seeded inputs,
and writes one .npz per case.  The committed files in tests/golden/ were made
with:

    make -C oracle && python tests/golden/make_golden.py --out tests/golden

(on a B200; the reference needs cuFFT and a GPU).  The CPU tests check the
oracle against these files; the GPU tests check the CUDA path against both.
"""
from __future__ import annotations

import argparse
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import ns3d_oracle as O  # noqa: E402
from oracle.ref_lib import RefSolver  # noqa: E402

CASES = {
    # name: (Nx, Ny, Nz, Lx, Ly, Lz, Re, dt, forcing wavenumber)
    "iso16": (16, 16, 16, 2 * math.pi, 2 * math.pi, 2 * math.pi, 50.0, 5e-3, 4),
    "aniso16x8x24": (16, 8, 24, 4 * math.pi, 2 * math.pi, math.pi, 80.0, 4e-3, 2),
}


def physical_rms(g, U):
    u = O.physical_velocity(g, U)
    return math.sqrt(sum(float(np.mean(a * a)) for a in u) / 3.0)


def odd_input(g, seed, kmax):
    """Pure-imaginary divergence-free field with O(1) physical amplitude."""
    P = O.random_perturbation(g, seed, kmin=1.0, kmax=kmax)
    s = 1.0 / physical_rms(g, P)
    return [s * p for p in P]


def general_input(g, seed, kmax):
    """General real field (complex coefficients), Hermitian on the kz=0/Nz/2 planes."""
    rng = np.random.Generator(np.random.PCG64(seed))
    m = g.m[:, None, None].astype(float)
    n = g.n[None, :, None].astype(float)
    q = g.q[None, None, :].astype(float)
    kk = np.sqrt(m * m + n * n + q * q)
    amp = np.where((kk >= 1) & (kk <= kmax), 1.0 / np.maximum(kk, 1.0), 0.0)
    jm = (-np.arange(g.Nx)) % g.Nx
    km = (-np.arange(g.Ny)) % g.Ny
    U = []
    for _ in range(3):
        w = (rng.standard_normal(g.shape_c) + 1j * rng.standard_normal(g.shape_c)) * amp
        for l in [0] + ([g.Nz // 2] if g.Nz % 2 == 0 else []):
            P = w[:, :, l]
            w[:, :, l] = 0.5 * (P + np.conj(P[jm][:, km]))
        w[0, 0, 0] = 0
        U.append(w)
    U = O.leray_project(g, U)
    s = 1.0 / physical_rms(g, U)
    return [s * u for u in U]


def stack(U):
    return np.stack([np.asarray(u) for u in U])


def run_case(name, out_dir):
    Nx, Ny, Nz, Lx, Ly, Lz, Re, dt, nf = CASES[name]
    g = O.Grid(Nx, Ny, Nz, Lx, Ly, Lz)
    kmax = min(Nx, Ny, Nz) / 3.0
    Uo = odd_input(g, 11, kmax)
    Vo = odd_input(g, 12, kmax)
    Ug = general_input(g, 13, kmax)
    F = O.kolmogorov_forcing(g, nf)
    rec = dict(Nx=Nx, Ny=Ny, Nz=Nz, Lx=Lx, Ly=Ly, Lz=Lz, Re=Re, dt=dt,
               U_odd=stack(Uo), V_odd=stack(Vo), U_gen=stack(Ug), F=stack(F))
    rng = np.random.Generator(np.random.PCG64(99))
    Xnh = rng.standard_normal(g.shape_c) + 1j * rng.standard_normal(g.shape_c)
    rec["X_nonherm"] = Xnh
    with RefSolver(Nx, Ny, Nz, Lx, Ly, Lz) as R:
        rec["c2r_nonherm"] = R.c2r(Xnh)
        R.set_f(F)
        R.set_u(Uo)
        rec["conv_odd"] = stack(R.conv())
        R.set_u(Ug)
        rec["conv_gen"] = stack(R.conv())
        R.set_u(Uo)
        R.set_v(Vo)
        rec["conv_uv"] = stack(R.conv_uv())
        R.set_u(Uo)
        rec["rhs_odd"] = stack(R.rhs(Re))
        R.set_u(Uo)
        R.euler(dt, Re)
        rec["euler_odd"] = stack(R.get_u())
        R.set_u(Uo)
        R.rk3(1, dt, Re)
        rec["rk3x1_odd"] = stack(R.get_u())
        R.set_u(Uo)
        R.rk3(5, dt, Re)
        rec["rk3x5_odd"] = stack(R.get_u())
        R.set_u(Ug)
        R.rk3(1, dt, Re)
        rec["rk3x1_gen"] = stack(R.get_u())
        R.set_u(Uo)
        R.set_v(Vo)
        R.jvp(1, dt, Re)
        rec["jvp_u"] = stack(R.get_u())
        rec["jvp_v"] = stack(R.get_v())
        R.set_u(Uo)
        R.set_v(Vo)
        R.linrhs(dt, Re)
        rec["linrhs_v"] = stack(R.get_v())
        R.set_u(Uo)
        R.set_v(Vo)
        R.iuv(dt, Re)
        rec["iuv_v"] = stack(R.get_v())
        R.set_u(Uo)
        e, d = R.diag()
        rec["diag_odd"] = np.array([e, d])
    path = os.path.join(out_dir, f"{name}.npz")
    np.savez_compressed(path, **rec)
    return path


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    ap.add_argument("--cases", nargs="*", default=list(CASES))
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    for c in a.cases:
        print("wrote", run_case(c, a.out))


if __name__ == "__main__":
    main()
