"""Golden vectors of the main loop's diagnostics from the reference's own
CUDA build: the 50-column time_dependant.dat record, the Helmholtz and
cut-off filtered velocities, the finite-difference curl and Shapiro's error
after a few RK3 steps (Source/NS3D_periodic.cu:1324-1452, Source/
math_support.cu:680-987, Source/Shapiro_test.cu:38-50), driven through
oracle/_ref/libns3d_ref.so.  The committed tests/golden/diagnostics.npz was
made on a B200 with

    make -C oracle && python tests/golden/make_golden_diag.py

The record is stored twice: "record" with the inverse transform applied to a
copy of the state, and "record_inplace" as main runs it, on the state arrays
themselves; cuFFT's out-of-place multi-dimensional complex-to-real transform
may overwrite its input (on B200 with cuFFT 12.9 it does), so there the
filtered and spectral columns read what the transform left behind;
"state_change_by_record" is the largest change it made to the state.
"""
from __future__ import annotations

import argparse
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, HERE):
    if p not in sys.path:
        sys.path.insert(0, p)

from oracle import ns3d_oracle as O  # noqa: E402
from oracle.ref_lib import RefSolver  # noqa: E402
from make_golden import general_input, stack  # noqa: E402

CASES = {
    # name: (Nx, Ny, Nz, Lx, Ly, Lz, Re, dt)
    "iso16": (16, 16, 16, 2 * math.pi, 2 * math.pi, 2 * math.pi, 50.0, 5e-3),
    "aniso16x8x24": (16, 8, 24, 4 * math.pi, 2 * math.pi, math.pi, 80.0, 4e-3),
    "iso32": (32, 32, 32, 2 * math.pi, 2 * math.pi, 2 * math.pi, 100.0, 4e-3),
}
SHAPIRO_STEPS = 20
SHAPIRO_RE = 10.0
SHAPIRO_DT = 0.02


def run_case(name):
    Nx, Ny, Nz, Lx, Ly, Lz, Re, dt = CASES[name]
    g = O.Grid(Nx, Ny, Nz, Lx, Ly, Lz)
    U = general_input(g, 21, min(Nx, Ny, Nz) / 3.0)
    rng = np.random.Generator(np.random.PCG64(22))
    u_phys = rng.standard_normal((3, Nx, Ny, Nz))
    out = {}
    with RefSolver(Nx, Ny, Nz, Lx, Ly, Lz) as R:
        R.set_f([np.zeros(g.shape_c, np.complex128)] * 3)
        # a state the reference stepped itself (non-Hermitian kz=0 plane parts included)
        R.set_u(U)
        R.rk3(3, dt, Re)
        S = R.get_u()
        out["U"] = stack(S)
        out["record"] = R.record(0.75, Re, preserve=True)
        R.set_u(S)
        out["record_inplace"] = R.record(0.75, Re, preserve=False)
        out["state_change_by_record"] = np.array(float(np.max(np.abs(stack(R.get_u()) - out["U"]))))
        R.set_u(S)
        if Nx * Ny * Nz <= 16 ** 3:  # the field-sized outputs only for the small grids
            out["filt_h1"], out["filt_c01"] = R.filters(1.0, 0.1)
            out["filt_h03"], out["filt_c025"] = R.filters(0.3, 0.25)
            out["u_phys"] = u_phys
            out["curl"] = R.curl(u_phys)
        if (Lx, Ly, Lz) == (2 * math.pi,) * 3:
            # Re and dt: the RK3 error of the decay (~1e-9) stands well above
            # rounding, and dt |k|^2_max / Re stays inside RK3's stability
            # interval for every mode of the grid
            R.set_u([R.r2c(a) for a in O.shapiro_physical(g, 0.0, SHAPIRO_RE)])
            R.rk3(SHAPIRO_STEPS, SHAPIRO_DT, SHAPIRO_RE)
            out["shapiro_U"] = stack(R.get_u())
            out["shapiro_error"] = np.array(R.shapiro_error(SHAPIRO_STEPS * SHAPIRO_DT,
                                                            SHAPIRO_RE))
    return dict(Nx=Nx, Ny=Ny, Nz=Nz, Lx=Lx, Ly=Ly, Lz=Lz, Re=Re, dt=dt, **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden", "diagnostics.npz"))
    a = ap.parse_args()
    rec = {}
    for name in CASES:
        for k, v in run_case(name).items():
            rec[f"{name}/{k}"] = v
    np.savez_compressed(a.out, **rec)
    print("wrote", a.out)


if __name__ == "__main__":
    main()
