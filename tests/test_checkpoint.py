"""Checkpoint files in the reference's wire format (Source/file_operations.cu):
this library's writer and reader against the reference's own, both ways,
byte for byte, including the reference's up-sampling of a coarser Fourier
file.  Host code on both sides: no GPU needed."""
import ctypes
import os

import numpy as np
import pytest

from ns3dperiodic_b200 import solver as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "libns3d_ref.so")
_dp = ctypes.POINTER(ctypes.c_double)


@pytest.fixture
def ref(tmp_path, monkeypatch):
    if not os.path.exists(REF):
        pytest.skip("oracle/_ref/libns3d_ref.so not built (needs the reference tree)")
    monkeypatch.chdir(tmp_path)  # the reference uses fixed names in the working directory
    lib = ctypes.CDLL(REF)
    for name in ("ref_write_control_fourier", "ref_read_control_fourier"):
        getattr(lib, name).argtypes = [ctypes.c_int] * 3 + [_dp]
    for name in ("ref_write_control_file", "ref_read_control_file"):
        getattr(lib, name).argtypes = [ctypes.c_int] * 3 + [_dp] * 3
    return lib


def _fields(shape, seed):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal(shape) + 1j * rng.standard_normal(shape) for _ in range(3)]


def _packed(U):
    return np.ascontiguousarray(np.stack(U)).view(np.float64)


def _ref_read_fourier(ref, Nx, Ny, Mz):
    out = np.zeros((3, Nx, Ny, Mz), dtype=np.complex128)
    ref.ref_read_control_fourier(Nx, Ny, Mz, out.view(np.float64).ctypes.data_as(_dp))
    return list(out)


def test_fourier_writer_is_byte_identical(ref, tmp_path):
    U = _fields((12, 8, 6), 1)
    ref.ref_write_control_fourier(12, 8, 6, _packed(U).ctypes.data_as(_dp))
    S.write_control_fourier(tmp_path / "ours.dat", U)
    assert (tmp_path / "ours.dat").read_bytes() == (tmp_path / "control_file_Fourier.dat").read_bytes()


def test_fourier_round_trips_both_ways(ref, tmp_path):
    U = _fields((16, 8, 9), 2)
    S.write_control_fourier("control_file_Fourier.dat", U)
    got = _ref_read_fourier(ref, 16, 8, 9)
    for a, b in zip(got, U):
        np.testing.assert_array_equal(a, b)
    ref.ref_write_control_fourier(16, 8, 9, _packed(U).ctypes.data_as(_dp))
    back, ext = S.read_control_fourier("control_file_Fourier.dat", 16, 8, 16)
    assert ext == (16, 8, 9)
    for a, b in zip(back, U):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("coarse,fine", [((8, 8, 8), (16, 16, 16)), ((16, 8, 16), (32, 16, 32))])
def test_coarse_fourier_file_is_upsampled_like_the_reference(ref, tmp_path, coarse, fine):
    (nx, ny, nz), (Nx, Ny, Nz) = coarse, fine
    U = _fields((nx, ny, nz // 2 + 1), 3)
    S.write_control_fourier("control_file_Fourier.dat", U)
    mine, ext = S.read_control_fourier("control_file_Fourier.dat", Nx, Ny, Nz)
    assert ext == (nx, ny, nz // 2 + 1)
    theirs = _ref_read_fourier(ref, Nx, Ny, Nz // 2 + 1)
    for a, b in zip(mine, theirs):
        np.testing.assert_array_equal(a, b)
    assert np.count_nonzero(mine[0]) == nx * ny * (nz // 2 + 1)


def test_physical_file_round_trips_both_ways(ref, tmp_path):
    rng = np.random.default_rng(4)
    u = [rng.standard_normal((8, 12, 16)) for _ in range(3)]
    S.write_control_file("control_file.dat", u)
    got = [np.zeros((8, 12, 16)) for _ in range(3)]
    ref.ref_read_control_file(8, 12, 16, *[g.ctypes.data_as(_dp) for g in got])
    for a, b in zip(got, u):
        np.testing.assert_array_equal(a, b)
    ours = (tmp_path / "control_file.dat").read_bytes()
    ref.ref_write_control_file(8, 12, 16, *[x.ctypes.data_as(_dp) for x in u])
    assert (tmp_path / "control_file.dat").read_bytes() == ours
    back = S.read_control_file("control_file.dat", 8, 12, 16)
    for a, b in zip(back, u):
        np.testing.assert_array_equal(a, b)


def test_unreadable_or_finer_files_are_errors(tmp_path):
    from ns3dperiodic_b200 import Ns3dError

    U = _fields((16, 16, 9), 5)
    S.write_control_fourier(tmp_path / "fine.dat", U)
    with pytest.raises(Ns3dError):  # a finer file than the target grid
        S.read_control_fourier(tmp_path / "fine.dat", 8, 8, 8)
    (tmp_path / "bad.dat").write_text("1.0 2.0 x 4.0 5.0 6.0\n")
    with pytest.raises(Ns3dError):
        S.read_control_fourier(tmp_path / "bad.dat", 8, 8, 8)
    (tmp_path / "odd.dat").write_text("1.0 2.0 3.0\n" * 7)
    with pytest.raises(Ns3dError):  # 7 lines match no grid
        S.read_control_fourier(tmp_path / "odd.dat", 8, 8, 8)
    with pytest.raises(Ns3dError):
        S.read_control_fourier(tmp_path / "missing.dat", 8, 8, 8)
