"""The FP32 precision mode (ns3d_set_precision): transforms and products in
FP32, state and update in FP64.  Checked against this library's FP64 path on
the same inputs and against Shapiro's exact solution; the FP64 path is
unchanged after switching back; ensembles and the server give the same FP32
results batched as alone.

Tolerances (FP32 rounding ~6e-8 relative, accumulated over the steps): one
RK3 step 1e-7 relative L2 to FP64; 50 steps of the Kolmogorov workload 1e-6;
20 tangent steps of a unit perturbation 1e-5 (the stated FP32 tolerance; the
perturbation has no exactly represented laminar part); the Shapiro run 1e-6
against the exact field (FP64 reaches 1e-10 there)."""
import math

import numpy as np
import pytest

from oracle import ns3d_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t

    if not t.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return t


def _h(F):
    return [f.cpu().numpy() for f in F]


@pytest.mark.parametrize("N", [32, 64, 96, 192])
def test_fp32_steps_track_fp64(torch, N):
    from ns3dperiodic_b200 import Solver
    from ns3dperiodic_b200 import workload as W

    Re = 200.0
    U0, F = W.kolmogorov_state(N, Re, 3, rel_amp=0.05)
    dt = W.kolmogorov_dt(N, Re)
    with Solver(N, N, N) as S:
        S.set_forcing(S.to_device(F))
        ref1 = _h(S.rk3_ssp(S.to_device(U0), dt, Re))
        ref50 = _h(S.rk3_ssp(S.to_device(U0), dt, Re, nsteps=50))
        S.precision = "fp32"
        assert S.precision == "fp32"
        one = _h(S.rk3_ssp(S.to_device(U0), dt, Re))
        fifty = _h(S.rk3_ssp(S.to_device(U0), dt, Re, nsteps=50))
        e1, e50 = O.rel_l2(one, ref1), O.rel_l2(fifty, ref50)
        assert 0.0 < e1 < 1e-7 and e50 < 1e-6, (e1, e50)
        S.precision = "fp64"
        again = _h(S.rk3_ssp(S.to_device(U0), dt, Re, nsteps=50))
        assert all(np.array_equal(a, b) for a, b in zip(again, ref50))


@pytest.mark.parametrize("N", [48, 96, 192])
def test_steps_are_deterministic_in_both_precisions(torch, N):
    """Repeated runs from the same state give the same bits: a race between
    the warps of a pass (for instance over a shared-memory slot) shows up as
    run-to-run differences long before it shows up as a wrong answer."""
    from ns3dperiodic_b200 import Solver
    from ns3dperiodic_b200 import workload as W

    Re = 200.0
    U0, F = W.kolmogorov_state(N, Re, 3, rel_amp=0.05)
    dt = W.kolmogorov_dt(N, Re)
    with Solver(N, N, N) as S:
        S.set_forcing(S.to_device(F))
        for prec in ("fp64", "fp32"):
            S.precision = prec
            runs = [_h(S.rk3_ssp(S.to_device(U0), dt, Re, nsteps=20)) for _ in range(3)]
            assert all(np.isfinite(u).all() for u in runs[0]), prec
            for r in runs[1:]:
                assert all(np.array_equal(a, b) for a, b in zip(r, runs[0])), prec


@pytest.mark.parametrize("N", [32, 128])
def test_fp32_in_place_update(torch, N):
    """single_time_step writes the new state over its input (the fwd_x update's
    output aliases the state it reads): the FP32 mode against the oracle's FP64
    Euler step from the same state, 1e-7 relative L2."""
    from ns3dperiodic_b200 import Solver
    from ns3dperiodic_b200 import workload as W

    Re = 200.0
    g = O.Grid(N, N, N)
    U0, F = W.kolmogorov_state(N, Re, 5, rel_amp=0.05)
    dt = W.kolmogorov_dt(N, Re)
    want = O.single_time_step(g, U0, F, dt, Re)
    with Solver(N, N, N) as S:
        S.precision = "fp32"
        S.set_forcing(S.to_device(F))
        U = S.to_device(U0)
        S.single_time_step(U, dt, Re)
        err = O.rel_l2(_h(U), want)
    assert 0.0 < err < 1e-7, err


def test_fp32_shapiro(torch):
    from ns3dperiodic_b200 import Solver

    g = O.Grid(32, 32, 32)
    Re, dt = 100.0, 1e-3
    with Solver(32, 32, 32) as S:
        S.precision = "fp32"
        U = S.rk3_ssp(S.to_device(O.shapiro_hat(g, 0.0, Re)), dt, Re, nsteps=100)
        err = O.rel_l2(_h(U), O.shapiro_hat(g, 100 * dt, Re))
        assert err < 1e-6, err
        assert float(np.max(np.abs(O.divergence_hat(g, _h(U))))) < 1e-6 * float(
            np.max(np.abs(_h(U)[0])))


def test_fp32_tangent_and_rhs_track_fp64(torch):
    from ns3dperiodic_b200 import Solver
    from ns3dperiodic_b200 import workload as W

    N, Re = 48, 100.0
    with Solver(N, N, N) as S:
        S.set_forcing(S.to_device(W.kolmogorov_forcing(N, N, N)))
        U, V = S.request_fields(Re, 9)
        u0, v0 = _h(U), _h(V)
        dt = W.kolmogorov_dt(N, Re)
        S.rk3_ssp_uv(U, V, dt, Re, nsteps=20)
        ref = _h(V)
        S.precision = "fp32"
        U2, V2 = S.to_device(u0), S.to_device(v0)
        S.rk3_ssp_uv(U2, V2, dt, Re, nsteps=20)
        assert O.rel_l2(_h(V2), ref) < 1e-5


def test_fp32_ensemble_equals_instances_alone(torch):
    from ns3dperiodic_b200 import Ensemble, Solver
    from ns3dperiodic_b200 import workload as W

    N, Res = 32, [80.0, 160.0, 320.0]
    states = [W.kolmogorov_state(N, Re, b, rel_amp=0.05) for b, Re in enumerate(Res)]
    E = Ensemble(len(Res), N, N, N)
    E.set_precision("fp32")
    E.set_forcing(states[0][1])
    E.set_params([W.kolmogorov_dt(N, Re) for Re in Res], Res)
    U = E.to_device([np.stack([st[0][c] for st in states]) for c in range(3)])
    E.rk3_steps(U, 6)
    with Solver(N, N, N) as S:
        S.precision = "fp32"
        S.set_forcing(S.to_device(states[0][1]))
        for b, Re in enumerate(Res):
            Ub = S.rk3_ssp(S.to_device(states[b][0]), W.kolmogorov_dt(N, Re), Re, nsteps=6)
            for c in range(3):
                assert torch.equal(U[c][b], Ub[c])
    E.close()


def test_fp32_server_result_equals_alone(torch):
    from ns3dperiodic_b200 import Server, Solver, request_steps
    from ns3dperiodic_b200 import workload as W

    with Server([16, 24], capacity=[2, 2]) as srv:
        srv.set_precision("fp32")
        reqs = [(16, 100.0, 0.05, 1), (24, 200.0, 0.04, 2), (16, 200.0, 0.03, 3)]
        first = srv.submit([(N, Re, T, sd, 0.0, 1) for N, Re, T, sd in reqs])
        assert srv.run() == 3
        for i, (N, Re, T, sd) in enumerate(reqs):
            with Solver(N, N, N) as S:
                S.precision = "fp32"
                S.set_forcing(S.to_device(W.kolmogorov_forcing(N, N, N)))
                U, V = S.request_fields(Re, sd)
                S.rk3_ssp_uv(U, V, W.kolmogorov_dt(N, Re), Re, nsteps=request_steps(N, Re, T))
                for a, b in zip(srv.result_field(first + i, N), _h(V)):
                    assert np.array_equal(a, b)
