"""Requests that bring their own fields (ns3d_server_submit_fields), the
exponential map served through the server (ns3d_map_exponential_served),
cancellation and the server's failure paths.

The work is what NSCallMatrixVector_exponential hands out per product
(Source/NS3D_periodic.cu:444-470): RK3_SSP_UV steps of a caller's base state
and tangent.  Checked bit for bit against the single-grid stepper
(ns3d_jvp_steps) and against ns3d_map_exponential, alone and in a mix with
other grids' requests.  Failure paths are made on the host: a NaN in one
request's submitted tangent, a capacity no device can hold, a cancelled
request; none of them faults the device."""
import math
import threading
import time

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


def _fields(N, Re, seed):
    """A caller's (u, v): Kolmogorov state and a unit perturbation (host)."""
    g = O.Grid(N, N, N)
    U, F = O.kolmogorov_state(g, Re, seed, rel_amp=0.05)
    V = O.random_perturbation(g, seed + 100)
    return g, U, V, F


def _solo(N, Re, dt, steps, U, V, F):
    """ns3d_jvp_steps on a single-grid handle: (u(T), v(T)) on the host."""
    from ns3dperiodic_b200 import Solver

    with Solver(N, N, N) as S:
        S.set_forcing(S.to_device(F))
        Ud, Vd = S.to_device(U), S.to_device(V)
        S.rk3_ssp_uv(Ud, Vd, dt, Re, nsteps=steps)
        return [x.cpu().numpy() for x in Ud], [x.cpu().numpy() for x in Vd]


def _dev(torch, F):
    return [torch.from_numpy(np.ascontiguousarray(f)).cuda() for f in F]


def _same(a, b):
    return all(np.array_equal(x, y) for x, y in zip(a, b))


def test_field_requests_equal_the_single_grid_stepper_alone_and_mixed(torch):
    from ns3dperiodic_b200 import Server

    cases = [(16, 40.0, 4e-3, 7, 1), (24, 80.0, 3e-3, 5, 2), (16, 60.0, 5e-3, 3, 3)]
    want = {}
    inputs = {}
    for N, Re, dt, steps, seed in cases:
        g, U, V, F = _fields(N, Re, seed)
        inputs[seed] = (U, V, F)
        want[seed] = _solo(N, Re, dt, steps, U, V, F)
    # alone: one request in the server
    N, Re, dt, steps, seed = cases[0]
    U, V, F = inputs[seed]
    with Server([16], capacity=[2]) as srv:
        Ud, Vd = _dev(torch, U), _dev(torch, V)
        Uo = [torch.empty_like(x) for x in Ud]
        rid = srv.submit_fields([dict(N=N, Re=Re, dt=dt, steps=steps, U=Ud, V=Vd, U_out=Uo)])
        assert srv.run() == 1
        r = srv.results()[rid]
        assert r["status"] == 0 and r["steps"] == steps
        assert _same([x.cpu().numpy() for x in Vd], want[seed][1])
        assert _same([x.cpu().numpy() for x in Uo], want[seed][0])
        assert _same([x.cpu().numpy() for x in Ud], U)  # U_out given: the input stays
        assert abs(r["v_norm"] - math.sqrt(sum(float(np.vdot(x, x).real)
                                              for x in want[seed][1]))) < 1e-12 * r["v_norm"]
    # mixed: field requests of two grids among seeded requests of a third
    with Server([16, 24, 32], capacity=[2, 1, 2]) as srv:
        srv.submit([(32, 100.0, 0.05, 9), (32, 200.0, 0.03, 10)])
        outs = {}
        reqs = []
        for N, Re, dt, steps, seed in cases:
            U, V, F = inputs[seed]
            Ud, Vd = _dev(torch, U), _dev(torch, V)
            outs[seed] = (Ud, Vd)
            reqs.append(dict(N=N, Re=Re, dt=dt, steps=steps, U=Ud, V=Vd, U_out=Ud))
        first = srv.submit_fields(reqs)
        assert srv.run() == 5
        res = srv.results()
        for i, (N, Re, dt, steps, seed) in enumerate(cases):
            assert res[first + i]["status"] == 0
            Ud, Vd = outs[seed]
            assert _same([x.cpu().numpy() for x in Vd], want[seed][1]), seed
            assert _same([x.cpu().numpy() for x in Ud], want[seed][0]), seed


def test_served_exponential_map_equals_the_plain_map(torch):
    """Arnoldi over the map served through the server equals Arnoldi over
    ns3d_map_exponential bit for bit (H, basis and the advanced base flow),
    alone and with other grids' requests waiting in the same server."""
    from ns3dperiodic_b200 import Krylov, Server, Solver

    N, Re, dt, steps, m = 16, 40.0, 5e-3, 2, 5
    g, U, _, F = _fields(N, Re, 7)
    f0 = np.random.default_rng(8).standard_normal(3 * N * N * (N // 2 + 1) - 3)

    def run(served, mixed=False):
        S = Solver(N, N, N)
        S.set_forcing(S.to_device(F))
        Ud, Vs = S.to_device(U), S.zeros()
        n = S.krylov_length
        kr = Krylov(n, m)
        srv = None
        if served:
            srv = Server([16, 24], capacity=[1, 2])
            if mixed:
                srv.submit([(24, 100.0, 0.05, 1), (24, 200.0, 0.04, 2), (24, 300.0, 0.03, 3)])
            A = kr.served_exponential_map(srv, S, Ud, Vs, dt, Re, steps)
        else:
            A = kr.exponential_map(S, Ud, Vs, dt, Re, steps)
        V = torch.zeros((m, n), dtype=torch.float64, device="cuda")
        H = np.zeros((m, m))
        f = torch.as_tensor(f0, device="cuda").clone()
        kr.arnoldi(A, V, H, f, 0, m)
        assert A.status == 0
        out = (H.copy(), V.cpu().numpy(), [x.cpu().numpy() for x in Ud])
        if served:
            assert A.ctx.requests >= m
            if mixed:
                srv.run()
                assert all(r["status"] == 0 for r in srv.results())
            srv.close()
        kr.close()
        S.close()
        return out

    plain = run(False)
    for mixed in (False, True):
        served = run(True, mixed)
        assert np.array_equal(served[0], plain[0]), mixed
        assert np.array_equal(served[1], plain[1]), mixed
        assert _same(served[2], plain[2]), mixed


def test_nan_in_one_request_leaves_the_others_unchanged(torch):
    from ns3dperiodic_b200 import Server

    N, Re, dt, steps = 16, 50.0, 4e-3, 4
    good = []
    for seed in (1, 2):
        g, U, V, F = _fields(N, Re, seed)
        good.append((U, V, _solo(N, Re, dt, steps, U, V, F)[1]))
    g, U, V, F = _fields(N, Re, 3)
    V[1][2, 3, 1] = complex(0.0, np.nan)  # planted in the submitted tangent
    with Server([N], capacity=[3]) as srv:
        reqs, outs = [], []
        for Uh, Vh in [(good[0][0], good[0][1]), (U, V), (good[1][0], good[1][1])]:
            Ud, Vd = _dev(torch, Uh), _dev(torch, Vh)
            outs.append(Vd)
            reqs.append(dict(N=N, Re=Re, dt=dt, steps=steps, U=Ud, V=Vd))
        first = srv.submit_fields(reqs)
        srv.run()
        res = srv.results()
    assert res[first + 1]["status"] == 5  # NS3D_ERR_NONFINITE
    assert res[first]["status"] == 0 and res[first + 2]["status"] == 0
    assert _same([x.cpu().numpy() for x in outs[0]], good[0][2])
    assert _same([x.cpu().numpy() for x in outs[2]], good[1][2])


def test_create_that_cannot_fit_returns_oom_and_frees_everything(torch):
    from ns3dperiodic_b200 import Server
    from ns3dperiodic_b200._lib import Ns3dError

    with Server([32, 64], capacity=[1, 1]):  # loads the kernels both grids use
        pass
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for caps in ([100000], [2, 100000]):  # the second grid fails after the first is built
        Ns = [64] if len(caps) == 1 else [32, 64]
        with pytest.raises(Ns3dError) as e:
            Server(Ns, capacity=caps)
        assert e.value.status == 3  # NS3D_ERR_OOM
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free0 - free1 < 64 << 20, (free0, free1)
    with Server([32], capacity=[2]) as srv:  # the device is still usable
        srv.submit([(32, 100.0, 0.02, 1)])
        assert srv.run() == 1


def test_cancel_frees_the_slot_for_the_next_arrival(torch):
    from ns3dperiodic_b200 import Server

    N, Re, dt = 16, 50.0, 4e-3
    g, U, V, F = _fields(N, Re, 4)
    want = _solo(N, Re, dt, 3, U, V, F)[1]
    with Server([N], capacity=[1]) as srv:
        Ua, Va = _dev(torch, U), _dev(torch, V)
        Ub, Vb = _dev(torch, U), _dev(torch, V)
        Vq = [torch.full_like(x, 7.0) for x in Vb]
        # A would run for seconds; the queued request writes into Vq
        ida = srv.submit_fields([dict(N=N, Re=Re, dt=dt, steps=30000, U=Ua, V=Va)])
        idq = srv.submit_fields([dict(N=N, Re=Re, dt=dt, steps=5, U=Ub, V=Vb, V_out=Vq)])
        idb = srv.submit_fields([dict(N=N, Re=Re, dt=dt, steps=3, U=Ub, V=Vb)])
        srv.run(max_seconds=0.2)  # A holds the only slot, the others wait
        res = srv.results()
        assert res[ida]["admitted"] >= 0 and res[idq]["admitted"] < 0
        srv.cancel(idq)  # queued: never starts
        # the running request, cancelled from another thread while run() runs
        th = threading.Thread(target=srv.run)
        th.start()
        time.sleep(0.3)
        srv.cancel(ida)
        th.join(timeout=120)
        assert not th.is_alive()
        res = srv.results()
        assert res[ida]["status"] == 8 and res[idq]["status"] == 8  # NS3D_ERR_CANCELLED
        assert res[idq]["admitted"] < 0
        assert res[idb]["status"] == 0
        assert res[idb]["admitted"] >= res[ida]["done"]
        assert _same([x.cpu().numpy() for x in Vb], want)
        with pytest.raises(Exception):
            srv.cancel(idb)  # finished
        with pytest.raises(Exception):
            srv.cancel(12345)  # unknown
        assert all(bool((x == 7.0).all()) for x in Vq)  # the cancelled request wrote nothing
