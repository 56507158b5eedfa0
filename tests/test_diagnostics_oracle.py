"""The oracle's restatement of the main loop's diagnostics against golden
vectors of the reference's own CUDA build (tests/golden/diagnostics.npz, made
by tests/golden/make_golden_diag.py), and the text formats of
time_dependant.dat and Ek.dat against the reference's writers.  CPU only.

Tolerances: record columns |a - b| <= 1e-12 max(1, |b|); filtered and curl
fields relative L2 <= 1e-13; Shapiro error absolute 1e-13 (the error is the
RK3 decay error, ~1e-9, far above rounding)."""
import ctypes
import os

import numpy as np
import pytest

from oracle import ns3d_oracle as O

CASES = ("iso16", "aniso16x8x24", "iso32")
SMALL = ("iso16", "aniso16x8x24")  # the cases with field-sized golden outputs
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "libns3d_ref.so")
COMPAT = os.path.join(ROOT, "ns3dperiodic_b200", "libns3d_compat.so")
_dp = ctypes.POINTER(ctypes.c_double)


def case(golden, name):
    d = golden["diagnostics"]
    get = lambda k: d[f"{name}/{k}"]  # noqa: E731
    g = O.Grid(int(get("Nx")), int(get("Ny")), int(get("Nz")), float(get("Lx")),
               float(get("Ly")), float(get("Lz")))
    return g, get


def close_cols(a, b, tol=1e-12):
    return np.abs(a - b) <= tol * np.maximum(1.0, np.abs(b))


@pytest.mark.parametrize("name", CASES)
def test_oracle_record_matches_reference(golden, name):
    g, get = case(golden, name)
    rec = O.series_record(g, list(get("U")), 0.75, float(get("Re")))
    ok = close_cols(rec, get("record"))
    assert ok.all(), np.nonzero(~ok)[0]


@pytest.mark.parametrize("name", CASES)
def test_in_place_record_of_main_reads_the_overwritten_state(golden, name):
    """main transforms the state arrays themselves; columns computed before
    anything reads the state again (1-22 and 29) are unaffected."""
    _, get = case(golden, name)
    same = np.r_[0:22, 28]
    assert close_cols(get("record_inplace")[same], get("record")[same]).all()
    changed = float(get("state_change_by_record"))
    if changed == 0.0:  # a cuFFT that keeps its input: all columns agree
        assert close_cols(get("record_inplace"), get("record")).all()


@pytest.mark.parametrize("name", SMALL)
def test_oracle_filters_match_reference(golden, name):
    g, get = case(golden, name)
    U = list(get("U"))
    for eps, rad, kh, kc in ((1.0, 0.1, "filt_h1", "filt_c01"),
                             (0.3, 0.25, "filt_h03", "filt_c025")):
        assert O.rel_l2(O.physical_velocity(g, O.helmholtz_filter(g, U, eps)), list(get(kh))) < 1e-13
        assert O.rel_l2(O.physical_velocity(g, O.cutoff_filter(g, U, rad)), list(get(kc))) < 1e-13


@pytest.mark.parametrize("name", SMALL)
def test_oracle_curl_matches_reference(golden, name):
    g, get = case(golden, name)
    assert O.rel_l2(O.curl_fd(g, list(get("u_phys"))), list(get("curl"))) < 1e-14


@pytest.mark.parametrize("name", ["iso16", "iso32"])
def test_oracle_shapiro_error_matches_reference(golden, name):
    g, get = case(golden, name)
    e = O.shapiro_error(g, list(get("shapiro_U")), 20 * 0.02, 10.0)
    ref = float(get("shapiro_error"))
    assert ref > 1e-10  # the RK3 decay error, not rounding
    assert abs(e - ref) <= 1e-13


def test_shapiro_field_is_an_exact_steady_beltrami_decay():
    g = O.Grid(16, 16, 16)
    U0 = O.shapiro_hat(g, 0.0, 2.0)
    U1 = O.shapiro_hat(g, 0.3, 2.0)
    s = np.exp(-3.0 * 0.3 / 2.0)
    assert O.rel_l2([s * u for u in U0], U1) < 1e-14
    assert float(np.max(np.abs(O.divergence_hat(g, U0)))) < 1e-9 * float(np.max(np.abs(U0[0])))


def _ref_lib():
    if not os.path.exists(REF):
        pytest.skip("oracle/_ref/libns3d_ref.so not built (needs the reference tree)")
    lib = ctypes.CDLL(REF)
    lib.ref_energy_spectrum.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        _dp]
    return lib


@pytest.mark.parametrize("name", CASES)
def test_energy_spectrum_text_matches_reference(golden, name, tmp_path):
    g, get = case(golden, name)
    U = np.ascontiguousarray(get("U"))
    lib = _ref_lib()
    path = tmp_path / "Ek_ref.dat"
    lib.ref_energy_spectrum(str(path).encode(), g.Nx, g.Ny, g.Mz,
                            U.view(np.float64).ctypes.data_as(_dp))
    ref = path.read_text().splitlines()
    ours = O.format_energy_spectrum(g, O.energy_spectrum(g, list(U))).splitlines()
    assert len(ours) == len(ref) == g.Nx // 2 + g.Ny // 2 + g.Mz
    for a, b in zip(ours, ref):
        fa, fb = a.split(), b.split()
        assert fa[0] == fb[0] and fa[2] == fb[2]
        assert abs(float(fa[1]) - float(fb[1])) <= 1e-13 * abs(float(fb[1]))


@pytest.mark.parametrize("name", CASES)
def test_compat_energy_spectrum_is_byte_identical(golden, name, tmp_path):
    g, get = case(golden, name)
    lib = _ref_lib()
    if not os.path.exists(COMPAT):
        pytest.skip("libns3d_compat.so not built")
    compat = ctypes.CDLL(COMPAT)
    fn = getattr(compat, "_Z25calculate_energy_spectrumPciiiPdS0_S0_S0_S0_S0_")
    fn.argtypes = [ctypes.c_char_p] + [ctypes.c_int] * 3 + [_dp] * 6
    U = np.ascontiguousarray(get("U"))
    parts = []
    for c in range(3):
        parts += [np.ascontiguousarray(U[c].real), np.ascontiguousarray(U[c].imag)]
    fn(str(tmp_path / "Ek_compat.dat").encode(), g.Nx, g.Ny, g.Mz,
       *[p.ctypes.data_as(_dp) for p in parts])
    lib.ref_energy_spectrum(str(tmp_path / "Ek_ref.dat").encode(), g.Nx, g.Ny, g.Mz,
                            U.view(np.float64).ctypes.data_as(_dp))
    assert (tmp_path / "Ek_compat.dat").read_bytes() == (tmp_path / "Ek_ref.dat").read_bytes()


def test_series_and_spectrum_writers_match_the_reference_formats(golden, tmp_path):
    from ns3dperiodic_b200 import solver as S

    g, get = case(golden, "iso16")
    recs = [get("record"), get("record_inplace")]
    with S.TimeSeries(tmp_path / "time_dependant.dat") as ts:
        for r in recs:
            ts.write(r)
    assert (tmp_path / "time_dependant.dat").read_text() == "".join(
        O.format_series_line(r) for r in recs)
    E = O.energy_spectrum(g, list(get("U")))
    S.write_energy_spectrum(tmp_path / "Ek.dat", g.Nx, g.Ny, g.Nz, E)
    assert (tmp_path / "Ek.dat").read_text() == O.format_energy_spectrum(g, E)
