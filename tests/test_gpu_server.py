"""The request server (ns3d_server_*): device-generated request fields, the
continuous-batching engine (admission by free slots, first come first served
per grid, arrival times, deadlines), and results that are bit for bit the
same in a mix as alone (the single-grid JVP stepper on the same fields)."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t

    if not t.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return t


def _dt(N, Re):
    return 0.3 * (2 * math.pi / N) / (Re / 16.0)


def test_request_fields_follow_the_recipe(torch):
    from ns3dperiodic_b200 import Solver
    from ns3dperiodic_b200 import workload as W

    N, Re = 32, 200.0
    with Solver(N, N, N) as S:
        U, V = S.request_fields(Re, 5)
        _, V2 = S.request_fields(Re, 5)
        _, V3 = S.request_fields(Re, 6)
    u, v = [x.cpu().numpy() for x in U], [x.cpu().numpy() for x in V]
    assert all(np.array_equal(a.cpu().numpy(), b) for a, b in zip(V2, v))  # deterministic
    assert not np.array_equal(V3[0].cpu().numpy(), v[0])
    assert abs(sum(float(np.vdot(x, x).real) for x in v) - 1.0) < 1e-13
    assert all(float(np.abs(x.real).max()) == 0.0 for x in v)  # pure imaginary
    m = np.where(np.arange(N) >= N // 2, np.arange(N) - N, np.arange(N)).astype(float)
    q = np.arange(N // 2 + 1).astype(float)
    K = (m[:, None, None], m[None, :, None], q[None, None, :])
    div = sum(K[i] * v[i] for i in range(3))
    assert float(np.abs(div).max()) < 1e-15
    kk = np.sqrt(K[0] ** 2 + K[1] ** 2 + K[2] ** 2)
    assert float(np.abs(v[0][(kk > 8) | (kk < 1)]).max()) == 0.0
    jm = (-np.arange(N)) % N
    for l in (0, N // 2):  # Hermitian planes (to rounding)
        P = v[1][:, :, l]
        assert float(np.abs(P - np.conj(P[jm][:, jm])).max()) <= 1e-15 * float(np.abs(P).max())
    F = W.kolmogorov_forcing(N, N, N)
    lam = F[0] * (Re / 16.0)
    pert = [u[0] - lam, u[1], u[2]]
    base = math.sqrt(float(np.vdot(lam, lam).real))
    amp = math.sqrt(sum(float(np.vdot(x, x).real) for x in pert))
    assert abs(amp / base - 1e-3) < 1e-12


def _solo(N, Re, T, seed):
    from ns3dperiodic_b200 import Solver, request_steps
    from ns3dperiodic_b200 import workload as W

    with Solver(N, N, N) as S:
        S.set_forcing(S.to_device(W.kolmogorov_forcing(N, N, N)))
        U, V = S.request_fields(Re, seed)
        S.rk3_ssp_uv(U, V, _dt(N, Re), Re, nsteps=request_steps(N, Re, T))
        return [x.cpu().numpy() for x in V]


def test_results_are_the_same_in_a_mix_as_alone(torch):
    from ns3dperiodic_b200 import Server

    reqs = [(16, 100.0, 0.08, 1), (24, 200.0, 0.05, 2), (16, 400.0, 0.02, 3),
            (32, 100.0, 0.06, 4), (24, 400.0, 0.03, 5), (16, 200.0, 0.05, 6),
            (32, 200.0, 0.02, 7), (16, 100.0, 0.04, 8)]
    with Server([16, 24, 32], capacity=[3, 2, 2]) as srv:
        first = srv.submit([(N, Re, T, seed, 0.0, 1) for N, Re, T, seed in reqs])
        assert srv.run() == len(reqs)
        res = srv.results()
        for i, (N, Re, T, seed) in enumerate(reqs):
            r = res[first + i]
            assert r["status"] == 0 and r["done"] >= r["admitted"] >= 0.0
            v = srv.result_field(first + i, N)
            solo = _solo(N, Re, T, seed)
            for a, b in zip(v, solo):
                assert np.array_equal(a, b), (i, N)
            norm = math.sqrt(sum(float(np.vdot(x, x).real) for x in solo))
            assert abs(r["v_norm"] - norm) <= 1e-12 * norm
    # the first request alone on a fresh server
    N, Re, T, seed = reqs[0]
    with Server([N], capacity=[1]) as srv:
        srv.submit([(N, Re, T, seed, 0.0, 1)])
        srv.run()
        for a, b in zip(srv.result_field(0, N), _solo(N, Re, T, seed)):
            assert np.array_equal(a, b)


def test_admission_respects_capacity_order_and_arrivals(torch):
    from ns3dperiodic_b200 import Server

    with Server([16], capacity=[2]) as srv:
        reqs = [(16, 100.0, 0.03 + 0.01 * i, 10 + i, 0.0) for i in range(5)]
        reqs.append((16, 100.0, 0.02, 99, 0.3))  # arrives later
        srv.submit(reqs)
        assert srv.run() == 6
        res = srv.results()
    spans = [(r["admitted"], r["done"]) for r in res]
    for a, _ in spans:
        assert sum(1 for b, e in spans if b <= a < e) <= 2
    adm = [r["admitted"] for r in res[:5]]
    assert adm == sorted(adm)  # first come, first served within the grid
    assert res[5]["admitted"] >= 0.3


def test_run_stops_at_its_deadline_and_resumes(torch):
    from ns3dperiodic_b200 import Ns3dError, Server

    with Server([32], capacity=[2]) as srv:
        srv.submit([(32, 100.0, 0.6, 1, 0.0), (32, 100.0, 0.6, 2, 0.0), (32, 100.0, 0.6, 3, 0.0)])
        n1 = srv.run(0.0)
        assert n1 == 0 and srv.results()[2]["admitted"] < 0.0
        n2 = srv.run()
        assert n1 + n2 == 3
        assert all(r["status"] == 0 for r in srv.results())
        with pytest.raises(Ns3dError):  # arrival order
            srv.submit([(32, 100.0, 0.1, 4, 5.0), (32, 100.0, 0.1, 5, 1.0)])
        with pytest.raises(Ns3dError):  # no such grid
            srv.submit([(48, 100.0, 0.1, 6, 10.0)])
