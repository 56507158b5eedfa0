"""Analytic pins of the oracle: Shapiro's Beltrami flow and laminar Kolmogorov."""
import math

import numpy as np

from oracle import ns3d_oracle as O


def test_shapiro_32_100_steps():
    """Shapiro test (Source/Shapiro_test.cu:8-50): exp(-3t/Re) decay, rel L2 < 1e-10."""
    g = O.Grid(32, 32, 32)
    Re, dt = 100.0, 1e-3
    U = O.shapiro_hat(g, 0.0, Re)
    F = [np.zeros(g.shape_c, complex) for _ in range(3)]
    for _ in range(100):
        U = O.rk3_ssp(g, U, F, dt, Re)
    E = O.shapiro_hat(g, 100 * dt, Re)
    assert O.rel_l2(U, E) < 1e-10
    # divergence at round-off relative to |k||u|
    umax = max(float(np.abs(u).max()) for u in U)
    assert float(np.abs(O.divergence_hat(g, U)).max()) < 1e-13 * umax


def test_kolmogorov_laminar_fixed_point():
    """u = (Re/16) sin(4y) x is an exact steady state under f = sin(4y) x."""
    g = O.Grid(16, 16, 16)
    Re = 40.0
    F = O.kolmogorov_forcing(g, 4)
    U = [F[0] * (Re / 16.0), np.zeros(g.shape_c, complex), np.zeros(g.shape_c, complex)]
    Q = O.convolution(g, U)
    assert max(float(np.abs(q).max()) for q in Q) < 1e-9
    R = O.return_rhs(g, U, F, Re)
    scale = float(np.abs(F[0]).max())
    assert max(float(np.abs(r).max()) for r in R) < 1e-12 * scale
    U1 = O.rk3_ssp(g, U, F, 0.01, Re)
    assert O.rel_l2(U1, U) < 1e-14


def test_mask_is_kz_prefix_for_all_extents():
    for n in (8, 16, 24, 32, 48, 64, 96, 128, 192, 256):
        qc = O.Grid(n, n, n).mask_cutoff()
        assert qc.min() >= 0 and qc.max() <= n // 2 + 1
