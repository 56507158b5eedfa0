"""Ensembles (ns3d_ensemble_*): instances of one grid stepped together give,
instance by instance and bit for bit, what ns3d_rk3_steps gives for each one
alone, with each instance's own dt and Re; several ensembles of different
grids on different streams run concurrently with the same results."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t

    if not t.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return t


def _instance(N, Re, seed):
    from ns3dperiodic_b200 import workload as W

    return W.kolmogorov_state(N, Re, seed, rel_amp=0.05)


def _dt(N, Re):
    from ns3dperiodic_b200 import workload as W

    return W.kolmogorov_dt(N, Re)


@pytest.mark.parametrize("N,B", [(32, 5), (48, 3), (64, 2)])
def test_ensemble_equals_instances_alone(torch, N, B):
    from ns3dperiodic_b200 import Ensemble, Solver

    Res = [50.0 + 90.0 * b for b in range(B)]
    states = [_instance(N, Re, b) for b, Re in enumerate(Res)]
    F = states[0][1]
    E = Ensemble(B, N, N, N)
    E.set_forcing(F)
    E.set_params([_dt(N, Re) for Re in Res], Res)
    U = E.to_device([np.stack([st[0][c] for st in states]) for c in range(3)])
    E.rk3_steps(U, 7)
    en, di = E.diagnostics(U)
    with Solver(N, N, N) as S:
        S.set_forcing(S.to_device(F))
        for b, Re in enumerate(Res):
            Ub = S.rk3_ssp(S.to_device(states[b][0]), _dt(N, Re), Re, nsteps=7)
            for c in range(3):
                assert torch.equal(U[c][b], Ub[c])
            e1, d1, _ = S.diagnostics(Ub)
            assert en[b] == e1 and di[b] == d1
    E.close()


def test_mixed_grids_on_streams_overlap_and_agree(torch):
    from ns3dperiodic_b200 import Ensemble

    groups = {32: [60.0, 120.0, 240.0], 48: [80.0, 400.0], 64: [150.0]}
    ens, fields, ref = [], [], []
    for N, Res in groups.items():
        states = [_instance(N, Re, 10 + b) for b, Re in enumerate(Res)]
        E = Ensemble(len(Res), N, N, N)
        E.set_forcing(states[0][1])
        E.set_params([_dt(N, Re) for Re in Res], Res)
        host = [np.stack([st[0][c] for st in states]) for c in range(3)]
        # the same ensemble alone, on its default stream
        U1 = E.to_device(host)
        E.rk3_steps(U1, 5)
        torch.cuda.synchronize()
        ref.append(U1)
        E.set_stream(torch.cuda.Stream())
        ens.append(E)
        fields.append(E.to_device(host))
    torch.cuda.synchronize()
    for E, U in zip(ens, fields):
        E.rk3_steps(U, 5)
    torch.cuda.synchronize()
    for U, R in zip(fields, ref):
        for c in range(3):
            assert torch.equal(U[c], R[c])
    for E in ens:
        E.close()


def test_ensemble_parameter_errors(torch):
    from ns3dperiodic_b200 import Ensemble, Ns3dError

    E = Ensemble(2, 16, 16, 16)
    U = E.zeros()
    with pytest.raises(Ns3dError):  # parameters first
        E.rk3_steps(U, 1)
    with pytest.raises(Ns3dError):
        E.set_params([0.01, -1.0], [10.0, 10.0])
    with pytest.raises(Ns3dError):
        E.set_params([0.01, 0.01], [10.0, float("nan")])
    E.set_params([0.01, 0.02], [10.0, 20.0])
    E.rk3_steps(U, 2)  # zero state stays zero without forcing
    assert all(float(u.abs().max()) == 0.0 for u in U)
    E.close()
