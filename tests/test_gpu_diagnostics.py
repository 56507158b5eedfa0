"""Filters, curl, the per-step record, the energy spectrum and Shapiro's
solution on the GPU through the C ABI, against the reference's own CUDA
build (tests/golden/diagnostics.npz) and the oracle; and the reference's
harness relinked on libns3d_compat.so.

Tolerances: record columns |a - b| <= 1e-12 max(1, |b|); spectral filters
relative L2 <= 1e-14, physical filtered fields and curls <= 1e-13; energy
spectrum bins relative 1e-13; Shapiro errors absolute 1e-13 (the errors
are the RK3 decay error, ~1e-9)."""
import math
import os

import numpy as np
import pytest

from oracle import ns3d_oracle as O

pytestmark = pytest.mark.gpu

CASES = ("iso16", "aniso16x8x24", "iso32")
SMALL = ("iso16", "aniso16x8x24")  # the cases with field-sized golden outputs


@pytest.fixture(scope="module")
def torch():
    import torch as t

    if not t.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return t


def case(golden, name):
    d = golden["diagnostics"]
    get = lambda k: d[f"{name}/{k}"]  # noqa: E731
    dims = (int(get("Nx")), int(get("Ny")), int(get("Nz")))
    box = (float(get("Lx")), float(get("Ly")), float(get("Lz")))
    return O.Grid(*dims, *box), dims, box, get


def close_cols(a, b, tol=1e-12):
    return np.abs(a - b) <= tol * np.maximum(1.0, np.abs(b))


def dev(torch, F):
    return [torch.as_tensor(np.ascontiguousarray(f)).cuda() for f in F]


def host(F):
    return [f.cpu().numpy() for f in F]


@pytest.mark.parametrize("name", CASES)
def test_record_matches_reference_and_oracle(torch, golden, name):
    from ns3dperiodic_b200 import Solver

    g, dims, box, get = case(golden, name)
    S = Solver(*dims, *box)
    U = dev(torch, get("U"))
    rec = S.record(U, 0.75, float(get("Re")))
    ok = close_cols(rec, get("record"))
    assert ok.all(), np.nonzero(~ok)[0]
    assert close_cols(rec, O.series_record(g, list(get("U")), 0.75, float(get("Re")))).all()
    # the state is read, not written
    assert all(np.array_equal(a, b) for a, b in zip(host(U), get("U")))
    S.close()


def test_time_series_file_follows_the_time_loop(torch, golden, tmp_path):
    from ns3dperiodic_b200 import Solver
    from ns3dperiodic_b200.solver import TimeSeries

    g, dims, box, get = case(golden, "iso16")
    Re, dt = float(get("Re")), float(get("dt"))
    S = Solver(*dims, *box)
    S.set_forcing(S.zeros())
    U = dev(torch, get("U"))
    recs = []
    with TimeSeries(tmp_path / "time_dependant.dat") as ts:
        for _ in range(3):
            S.rk3_ssp(U, dt, Re)
            recs.append(ts.step(S, U, dt, Re))
    lines = (tmp_path / "time_dependant.dat").read_text().splitlines()
    assert len(lines) == 3
    for i, (line, r) in enumerate(zip(lines, recs)):
        vals = np.array([float(x) for x in line.split(" ")])
        assert vals.size == 50
        assert line + "\n" == O.format_series_line(r)
        assert math.isclose(vals[0], 2 * dt * (i + 1), rel_tol=1e-6)
    S.close()


@pytest.mark.parametrize("name", SMALL)
def test_filters_match_reference(torch, golden, name):
    from ns3dperiodic_b200 import Solver

    g, dims, box, get = case(golden, name)
    S = Solver(*dims, *box)
    Uh = list(get("U"))
    U = dev(torch, Uh)
    for eps, rad, kh, kc in ((1.0, 0.1, "filt_h1", "filt_c01"),
                             (0.3, 0.25, "filt_h03", "filt_c025")):
        fh = S.helmholtz_filter(U, eps)
        fc = S.cutoff_filter(U, rad)
        assert O.rel_l2(host(fh), O.helmholtz_filter(g, Uh, eps)) < 1e-14
        assert O.rel_l2(host(fc), O.cutoff_filter(g, Uh, rad)) < 1e-14
        assert O.rel_l2([S.ifftn(f).cpu().numpy() for f in fh], list(get(kh))) < 1e-13
        assert O.rel_l2([S.ifftn(f).cpu().numpy() for f in fc], list(get(kc))) < 1e-13
    # in place
    V = [u.clone() for u in U]
    S.cutoff_filter(V, 0.25, out=V)
    assert O.rel_l2(host(V), O.cutoff_filter(g, Uh, 0.25)) < 1e-14
    S.close()


@pytest.mark.parametrize("name", SMALL)
def test_curl_matches_reference(torch, golden, name):
    from ns3dperiodic_b200 import Solver

    g, dims, box, get = case(golden, name)
    S = Solver(*dims, *box)
    r = S.curl(dev(torch, get("u_phys")))
    assert O.rel_l2(host(r), list(get("curl"))) < 1e-13
    S.close()


@pytest.mark.parametrize("name", CASES)
def test_energy_spectrum_matches_oracle(torch, golden, name, tmp_path):
    from ns3dperiodic_b200 import Ns3dError, Solver

    g, dims, box, get = case(golden, name)
    S = Solver(*dims, *box)
    U = dev(torch, get("U"))
    E = S.energy_spectrum(U)
    Eo = O.energy_spectrum(g, list(get("U")))
    assert np.all(np.abs(E - Eo) <= 1e-13 * np.abs(Eo) + 1e-300)
    S.write_energy_spectrum(tmp_path / "Ek.dat", U)
    lines = (tmp_path / "Ek.dat").read_text().splitlines()
    ref = O.format_energy_spectrum(g, Eo).splitlines()
    for a, b in zip(lines, ref):
        fa, fb = a.split(), b.split()
        assert fa[0] == fb[0] and fa[2] == fb[2]
        assert abs(float(fa[1]) - float(fb[1])) <= 1e-13 * abs(float(fb[1]))
    with pytest.raises(Ns3dError):
        S._check(S._L.ns3d_energy_spectrum(S._h, *S._fields(U, "U"), E.ctypes.data, 3), "x")
    S.close()


@pytest.mark.parametrize("name", ["iso16", "iso32"])
def test_shapiro_solution_and_error(torch, golden, name):
    from ns3dperiodic_b200 import Solver

    g, dims, box, get = case(golden, name)
    S = Solver(*dims, *box)
    W = S.shapiro_state(0.0, 10.0)
    assert O.rel_l2(host(W), O.shapiro_hat(g, 0.0, 10.0)) < 1e-14
    ref = float(get("shapiro_error"))
    assert abs(S.shapiro_error(dev(torch, get("shapiro_U")), 0.4, 10.0) - ref) <= 1e-13
    S.set_forcing(S.zeros())
    S.rk3_ssp(W, 0.02, 10.0, nsteps=20)
    assert abs(S.shapiro_error(W, 0.4, 10.0) - ref) <= 1e-13
    S.close()


@pytest.mark.parametrize("name", CASES)
def test_reference_harness_relinked_on_compat_layer(torch, golden, name):
    """get_curl, the two filters, Image_to_Domain and the reductions of the
    record come from libns3d_compat.so here."""
    from oracle.ref_lib import COMPAT_LIB_PATH, RefSolver

    if not os.path.exists(COMPAT_LIB_PATH):
        pytest.skip("oracle/_ref/libns3d_ref_compat.so not built")
    g, dims, box, get = case(golden, name)
    with RefSolver(*dims, *box, lib_path=COMPAT_LIB_PATH) as R:
        R.set_f([np.zeros(g.shape_c, np.complex128)] * 3)
        R.set_u(list(get("U")))
        assert close_cols(R.record(0.75, float(get("Re")), preserve=False), get("record")).all()
        if name in SMALL:
            ph, pc = R.filters(1.0, 0.1)
            assert O.rel_l2(list(ph), list(get("filt_h1"))) < 1e-13
            assert O.rel_l2(list(pc), list(get("filt_c01"))) < 1e-13
            assert O.rel_l2(list(R.curl(get("u_phys"))), list(get("curl"))) < 1e-13
        if name != "aniso16x8x24":
            R.set_u(list(get("shapiro_U")))
            ref = float(get("shapiro_error"))
            assert abs(R.shapiro_error(0.4, 10.0) - ref) <= 1e-13
