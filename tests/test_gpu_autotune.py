"""Autotuner of the pass tiles (ns3d_autotune, ns3d_get/set_tiles): every
tile gives the default's result to round-off (the transforms only reorder
their floating-point operations), the tuner keeps what it measured, caches
per geometry, and an ensemble with tuned tiles still equals its instances
stepped alone with the same tiles, bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ONES = [1, 1, 1, 1]


@pytest.fixture(scope="module")
def torch():
    import torch as t

    if not t.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return t


def _state(shape, Re, seed):
    from ns3dperiodic_b200 import workload as W

    Nx, Ny, Nz = shape
    if Nx == Ny == Nz:
        return W.kolmogorov_state(Nx, Re, seed, rel_amp=0.05)
    rng = np.random.default_rng(seed)
    Mz = Nz // 2 + 1
    U = [1j * rng.standard_normal((Nx, Ny, Mz)) * 1e-2 * Nx * Ny * Nz for _ in range(3)]
    for u in U:
        u[0, 0, 0] = 0.0
    return U, [np.zeros_like(U[0]) for _ in range(3)]


def _rel(a, b, torch):
    num = sum(float(torch.linalg.vector_norm(x - y)) ** 2 for x, y in zip(a, b))
    den = sum(float(torch.linalg.vector_norm(y)) ** 2 for y in b)
    return (num / den) ** 0.5


def _alt_tiles(shape):
    Nx, Ny, _ = shape

    def alt(n):
        return n >= 48 if n % 3 == 0 else n >= 32

    return [int(alt(Nx)), int(alt(Ny)), int(alt(Ny)), int(alt(Nx))]


@pytest.mark.parametrize("shape", [(32, 32, 32), (48, 48, 48), (64, 64, 64), (128, 128, 128),
                                   (512, 8, 8), (8, 512, 8), (384, 8, 16), (256, 32, 8)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_alternative_tiles_match_the_default(torch, shape, precision):
    from ns3dperiodic_b200 import Solver

    Re, dt = 200.0, 1.0e-3
    U0, F = _state(shape, Re, 3)
    out = []
    for tiles in ([0, 0, 0, 0], _alt_tiles(shape)):
        with Solver(*shape) as S:
            S.precision = precision
            S.tiles = tiles
            assert S.tiles == tiles
            S.set_forcing(S.to_device(F))
            U = S.rk3_ssp(S.to_device(U0), dt, Re, nsteps=3)
            V = S.to_device([0.5 * u for u in U0])
            Uj, Vj = S.rk3_ssp_uv(S.to_device(U0), V, dt, Re, nsteps=2)
            out.append((U, Vj))
    tol = 1e-12 if precision == "fp64" else 2e-6
    assert _rel(out[1][0], out[0][0], torch) < tol
    assert _rel(out[1][1], out[0][1], torch) < tol


@pytest.mark.parametrize("shape", [(8, 192, 8), (16, 256, 16), (8, 384, 16), (8, 512, 8),
                                   (24, 256, 24), (16, 64, 24), (8, 48, 8), (8, 128, 16)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_bulk_copy_inv_y_matches_the_default(torch, shape, precision):
    """inv_y's tile 2: one thread per CTA loads each field's box of lines with
    a tensor copy (FP64; the FP32 mode and the tangent form run per-thread
    copies at the same points per thread).  Odd Mz leaves a last group of
    lines past the end of each x plane (filled with zeros by the copy, not
    stored); 384 takes each box in two copies of 192 rows."""
    from ns3dperiodic_b200 import Solver

    Re, dt = 200.0, 1.0e-3
    U0, F = _state(shape, Re, 5)
    out = []
    for tiles in ([0, 0, 0, 0], [0, 2, 0, 0]):
        with Solver(*shape) as S:
            S.precision = precision
            S.tiles = tiles
            assert S.tiles == tiles
            S.set_forcing(S.to_device(F))
            U = S.rk3_ssp(S.to_device(U0), dt, Re, nsteps=3)
            V = S.to_device([0.5 * u for u in U0])
            Uj, Vj = S.rk3_ssp_uv(S.to_device(U0), V, dt, Re, nsteps=2)
            S.synchronize()  # NS3D_ERR_TIMEOUT if a bounded wait gave up
            out.append((U, Vj))
    tol = 1e-12 if precision == "fp64" else 2e-6
    assert _rel(out[1][0], out[0][0], torch) < tol
    assert _rel(out[1][1], out[0][1], torch) < tol


def _rev_tiles(S):
    """Per family the first of tiles 3, 4 the handle accepts (0: neither)."""
    from ns3dperiodic_b200._lib import Ns3dError

    out = [0, 0, 0, 0]
    for f in range(3):  # inv_x, inv_y, fwd_y
        for tile in (3, 4):
            trial = list(out)
            trial[f] = tile
            try:
                S.tiles = trial
            except Ns3dError:
                continue
            out[f] = tile
            break
    S.tiles = [0, 0, 0, 0]
    return out


@pytest.mark.parametrize("shape", [(32, 32, 32), (48, 48, 48), (128, 128, 128), (24, 24, 24),
                                   (512, 8, 8), (8, 512, 8), (384, 8, 16), (8, 192, 8),
                                   (256, 32, 8)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_reversed_radix_schedules_match_the_default(torch, shape, precision):
    """Tiles 3 and 4: the radices of a line transform in reverse order (other
    first-exchange stride, padding and stage twiddles), same result to
    round-off."""
    from ns3dperiodic_b200 import Solver

    Re, dt = 200.0, 1.0e-3
    U0, F = _state(shape, Re, 11)
    out = []
    with Solver(*shape) as S:
        rev = _rev_tiles(S)
    assert any(rev), shape
    alt = _alt_tiles(shape)
    rev_alt = [4 if (f < 3 and alt[f]) else 0 for f in range(4)]
    for tiles in ([0, 0, 0, 0], rev, rev_alt):
        with Solver(*shape) as S:
            S.precision = precision
            try:
                S.tiles = tiles
            except Exception:
                assert tiles is rev_alt  # an alternative tile without a reversed order
                continue
            S.set_forcing(S.to_device(F))
            U = S.rk3_ssp(S.to_device(U0), dt, Re, nsteps=3)
            V = S.to_device([0.5 * u for u in U0])
            Uj, Vj = S.rk3_ssp_uv(S.to_device(U0), V, dt, Re, nsteps=2)
            out.append((U, Vj))
    tol = 1e-12 if precision == "fp64" else 2e-6
    for o in out[1:]:
        assert _rel(o[0], out[0][0], torch) < tol
        assert _rel(o[1], out[0][1], torch) < tol


def test_bulk_copy_ensemble_equals_instances_alone(torch):
    """The tensor maps cover every instance of a batch as x planes."""
    from ns3dperiodic_b200 import Ensemble, Solver
    from ns3dperiodic_b200 import workload as W

    shape, Res = (8, 256, 8), [80.0, 160.0, 320.0]
    states = [_state(shape, Re, 7 + b) for b, Re in enumerate(Res)]
    E = Ensemble(len(Res), *shape)
    E.tiles = [0, 2, 0, 0]
    E.set_forcing(states[0][1])
    E.set_params([1.0e-3] * len(Res), Res)
    U = E.to_device([np.stack([st[0][c] for st in states]) for c in range(3)])
    E.rk3_steps(U, 4)
    with Solver(*shape) as S:
        S.tiles = [0, 2, 0, 0]
        S.set_forcing(S.to_device(states[0][1]))
        for b, Re in enumerate(Res):
            Ub = S.rk3_ssp(S.to_device(states[b][0]), 1.0e-3, Re, nsteps=4)
            for c in range(3):
                assert torch.equal(U[c][b], Ub[c])
    E.close()


def test_autotune_keeps_what_it_measured_and_caches(torch):
    from ns3dperiodic_b200 import Solver

    with Solver(64, 64, 64) as S:
        r = S.autotune(reps=10, force=True)
        assert r["ms"] is not None and len(r["ms"]) == 4
        for f, times in enumerate(r["ms"]):
            assert 0 in times and 1 in times and all(x > 0.0 for x in times.values())
            fastest = min(times, key=times.get)
            want = fastest if times[fastest] < 0.98 * times[0] else 0
            assert r["tiles"][f] == want
        assert set(r["ms"][3]) == {0, 1}                     # fwd_x: two tiles
        assert set(r["ms"][0]) == {0, 1, 3}                  # 64: 16.4 reverses, 8.8 does not
        assert set(r["ms"][1]) == {0, 1, 2, 3}               # inv_y adds the bulk copy
        assert S.tiles == r["tiles"]
        with Solver(64, 64, 64) as S2:
            r2 = S2.autotune()
            assert r2["ms"] is None and r2["tiles"] == r["tiles"]
    with Solver(16, 16, 16) as S:  # no alternative tile below 32
        r = S.autotune(reps=3, force=True)
        assert r["tiles"] == [0, 0, 0, 0]
        assert all(set(times) == {0} for times in r["ms"])


def test_autotune_times_the_bulk_copy_tile(torch):
    """inv_y's bulk-copy tile is timed with the others and kept where it is
    the fastest and 2% faster than the default."""
    from ns3dperiodic_b200 import Solver

    with Solver(16, 256, 16) as S:
        r = S.autotune(reps=5, force=True)
        times = r["ms"][1]
        assert set(times) == {0, 1, 2, 4}  # 256: 16.16 has no reversed order
        fastest = min(times, key=times.get)
        want = fastest if times[fastest] < 0.98 * times[0] else 0
        assert r["tiles"][1] == want and S.tiles == r["tiles"]
        S.precision = "fp32"  # FP32 lines have no bulk-copy form to time
        r = S.autotune(reps=3, force=True)
        assert set(r["ms"][1]) == {0, 1, 4} and r["tiles"][1] != 2


def test_set_tiles_rejects_what_the_extent_lacks(torch):
    from ns3dperiodic_b200 import Solver
    from ns3dperiodic_b200._lib import Ns3dError

    with Solver(16, 32, 16) as S:
        with pytest.raises(Ns3dError):
            S.tiles = [0, 2, 0, 0]   # 32-point y lines never span 8 threads: no bulk copy
    with Solver(16, 64, 16) as S:
        with pytest.raises(Ns3dError):
            S.tiles = [1, 0, 0, 0]  # x = 16 has no alternative
        with pytest.raises(Ns3dError):
            S.tiles = [0, 0, 2, 0]   # only inv_y has a tile 2
        with pytest.raises(Ns3dError):
            S.tiles = [3, 0, 0, 0]   # x = 16: the 16-point radix has no other order
        with pytest.raises(Ns3dError):
            S.tiles = [0, 4, 0, 0]   # y = 64, 8 points: 8.8 reads the same reversed
        with pytest.raises(Ns3dError):
            S.tiles = [0, 0, 0, 3]   # fwd_x has no reversed schedules
        with pytest.raises(Ns3dError):
            S.tiles = [0, 5, 0, 0]
        S.tiles = [0, 1, 1, 0]       # y = 64 has one
        assert S.tiles == [0, 1, 1, 0]
        S.tiles = [0, 3, 3, 0]       # and 16.4 reverses to 4.16
        assert S.tiles == [0, 3, 3, 0]


def test_tiles_follow_the_precision(torch):
    from ns3dperiodic_b200 import Solver

    with Solver(32, 32, 32) as S:
        S.tiles = ONES
        S.precision = "fp32"
        assert S.tiles == [0, 0, 0, 0]
        S.tiles = [1, 0, 1, 0]
        S.precision = "fp64"
        assert S.tiles == ONES
        S.precision = "fp32"
        assert S.tiles == [1, 0, 1, 0]


def test_tuned_ensemble_equals_its_instances_alone(torch):
    from ns3dperiodic_b200 import Ensemble, Solver
    from ns3dperiodic_b200 import workload as W

    N, Res = 48, [80.0, 160.0, 320.0]
    states = [W.kolmogorov_state(N, Re, b, rel_amp=0.05) for b, Re in enumerate(Res)]
    E = Ensemble(len(Res), N, N, N)
    E.autotune(reps=5, force=True)
    E.tiles = ONES
    E.set_forcing(states[0][1])
    E.set_params([W.kolmogorov_dt(N, Re) for Re in Res], Res)
    U = E.to_device([np.stack([st[0][c] for st in states]) for c in range(3)])
    E.rk3_steps(U, 5)
    with Solver(N, N, N) as S:
        S.tiles = ONES
        S.set_forcing(S.to_device(states[0][1]))
        for b, Re in enumerate(Res):
            Ub = S.rk3_ssp(S.to_device(states[b][0]), W.kolmogorov_dt(N, Re), Re, nsteps=5)
            for c in range(3):
                assert torch.equal(U[c][b], Ub[c])
    E.close()


def test_changing_tiles_recaptures_the_step(torch):
    """The cached RK3 step graph holds the kernels of the tiles it was
    captured with: after set_tiles the step uses the new ones."""
    from ns3dperiodic_b200 import Solver
    from ns3dperiodic_b200 import workload as W

    N, Re = 64, 200.0
    U0, F = W.kolmogorov_state(N, Re, 1, rel_amp=0.05)
    dt = W.kolmogorov_dt(N, Re)
    with Solver(N, N, N) as S, Solver(N, N, N) as T:
        for X in (S, T):
            X.set_forcing(X.to_device(F))
        T.tiles = ONES
        S.rk3_ssp(S.to_device(U0), dt, Re, nsteps=2)  # captures the default step
        S.tiles = ONES
        a = S.rk3_ssp(S.to_device(U0), dt, Re, nsteps=2)
        b = T.rk3_ssp(T.to_device(U0), dt, Re, nsteps=2)
        for c in range(3):
            assert torch.equal(a[c], b[c])


def test_server_autotune_runs_between_runs(torch):
    """Tuned server grids give the single-grid result to round-off."""
    import math

    from ns3dperiodic_b200 import Server, Solver, request_steps
    from ns3dperiodic_b200 import workload as W

    N, Re, T, seed = 64, 100.0, 0.05, 7
    with Server([N], capacity=[2]) as srv:
        srv.autotune(reps=3)
        first = srv.submit([(N, Re, T, seed, 0.0, 1)])
        assert srv.run() == 1
        v = srv.result_field(first, N)
    with Solver(N, N, N) as S:
        S.set_forcing(S.to_device(W.kolmogorov_forcing(N, N, N)))
        U, V = S.request_fields(Re, seed)
        dt = 0.3 * (2.0 * math.pi / N) / (Re / 16.0)
        S.rk3_ssp_uv(U, V, dt, Re, nsteps=request_steps(N, Re, T))
        ref = [x.cpu().numpy() for x in V]
    num = sum(float(np.linalg.norm(a - b)) ** 2 for a, b in zip(v, ref))
    den = sum(float(np.linalg.norm(b)) ** 2 for b in ref)
    assert math.sqrt(num / den) < 1e-12
