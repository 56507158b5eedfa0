"""The C-ABI library: it loads, exports every symbol include/ns3d.h declares,
and its host-only helpers agree with the oracle.  No GPU needed."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

from oracle import ns3d_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ns3d.h")


def _declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ns3d_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    from ns3dperiodic_b200 import _lib

    lib = _lib.lib()
    declared = _declared()
    assert len(declared) >= 25
    for name in declared:
        assert hasattr(lib, name), name
    assert set(_lib.EXPORTS) == set(declared)


def test_missing_library_fails_loudly(monkeypatch):
    from ns3dperiodic_b200 import _lib

    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", "/nonexistent/libns3d_b200.so")
    with pytest.raises(_lib.Ns3dLibraryError):
        _lib.lib()


def test_supported_extents():
    from ns3dperiodic_b200 import supported_extent

    for n in (8, 16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512):
        assert supported_extent(n)
    for n in (0, 10, 100, 1024, -8):
        assert not supported_extent(n)


GRIDS = [
    (16, 16, 16, 2 * math.pi, 2 * math.pi, 2 * math.pi),
    (16, 8, 24, 4 * math.pi, 2 * math.pi, math.pi),
    (128, 128, 128, 2 * math.pi, 2 * math.pi, 2 * math.pi),
    (48, 96, 64, 1.0, 2.0, 3.0),
    (256, 192, 384, 2 * math.pi, 3.0, 5.0),
    (512, 512, 512, 2 * math.pi, 2 * math.pi, 2 * math.pi),
]


@pytest.mark.parametrize("grid", GRIDS)
def test_mask_cutoff_matches_reference_mask(grid):
    from ns3dperiodic_b200 import _lib

    Nx, Ny, Nz, Lx, Ly, Lz = grid
    q = np.zeros(Nx * Ny, np.uint16)
    rc = _lib.lib().ns3d_mask_cutoff(Nx, Ny, Nz, Lx, Ly, Lz, q.ctypes.data)
    assert rc == 0
    g = O.Grid(Nx, Ny, Nz, Lx, Ly, Lz)
    assert np.array_equal(q.reshape(Nx, Ny).astype(np.int32), g.mask_cutoff())


@pytest.mark.parametrize("n", [8, 24, 96, 256, 384, 512])
def test_twiddles(n):
    from ns3dperiodic_b200 import _lib

    t = np.zeros(2 * n)
    assert _lib.lib().ns3d_twiddles(n, t.ctypes.data) == 0
    e = np.arange(n)
    w = t[0::2] + 1j * t[1::2]
    assert np.max(np.abs(w - np.exp(2j * np.pi * e / n))) < 3e-15
    # exact quarter-wave values
    for q in range(4):
        if (q * n) % 4 == 0:
            assert w[q * n // 4] == [1, 1j, -1, -1j][q]


def test_bad_arguments_are_rejected_without_gpu():
    from ns3dperiodic_b200 import _lib

    lib = _lib.lib()
    h = ctypes.c_void_p()
    assert lib.ns3d_create(100, 64, 64, 1.0, 1.0, 1.0, ctypes.byref(h)) == 2  # unsupported
    assert lib.ns3d_create(64, 64, 64, -1.0, 1.0, 1.0, ctypes.byref(h)) == 1
    assert lib.ns3d_create(0, 64, 64, 1.0, 1.0, 1.0, ctypes.byref(h)) == 1
    assert lib.ns3d_destroy(None) == 1
    assert lib.ns3d_status_string(2) == b"unsupported grid extent"
