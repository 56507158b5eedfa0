"""The allocation-free nonlinear term, ns3d_convolution_noalloc.

It exists for callers that cannot allocate device memory on the call path:
programs that reserve all device memory up front for their own pool, callers
that keep no handle between calls, and code that cannot take the
synchronisation cudaMalloc/cudaFree may cost.  It must give the same result as
the handle-based ns3d_convolution while working only in the scratch array
compiled into the library.

This file is collected last on purpose (a failure here stops an -x run only
after every other test has run); it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative L2, the tolerance of the other GPU parity tests


def _field(shape, seed):
    """A real velocity field's half spectrum: Hermitian on the kz=0 / Nz/2 planes."""
    Nx, Ny, Mz = shape
    Nz = 2 * (Mz - 1)
    rng = np.random.Generator(np.random.PCG64(seed))
    jm = (-np.arange(Nx)) % Nx
    km = (-np.arange(Ny)) % Ny
    out = []
    for _ in range(3):
        w = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        for l in (0, Nz // 2):
            P = w[:, :, l]
            w[:, :, l] = 0.5 * (P + np.conj(P[jm][:, km]))
        w[0, 0, 0] = 0
        out.append(w)
    return out


def _rel(a, b):
    num = sum(float((x - y).abs().pow(2).sum()) for x, y in zip(a, b))
    den = sum(float(y.abs().pow(2).sum()) for y in b)
    return (num / den) ** 0.5


def _noalloc(lib, grid, U, Q, stream=None):
    Nx, Ny, Nz, Lx, Ly, Lz = grid
    return lib.ns3d_convolution_noalloc(Nx, Ny, Nz, Lx, Ly, Lz,
                                        *[ctypes.c_void_p(u.data_ptr()) for u in U],
                                        *[ctypes.c_void_p(q.data_ptr()) for q in Q],
                                        ctypes.c_void_p(stream))


def test_noalloc_convolution_matches_handle_entry_point_twice():
    import torch

    from ns3dperiodic_b200 import Solver, _lib

    lib = _lib.lib()
    grid = (32, 24, 48, 2 * np.pi, 3.0, 5.0)
    Nx, Ny, Nz = grid[:3]
    with Solver(*grid) as S:
        shape = S.shape
        assert Nx * Ny * (Nz // 2 + 1) <= 135168
        for call, seed in enumerate((1, 2)):  # two calls in a row, different inputs
            U = S.to_device(_field(shape, seed))
            want = S.calculate_convolution_2p3(U)
            got = [torch.full(shape, complex(np.nan, np.nan), dtype=torch.complex128,
                              device=S.device) for _ in range(3)]
            torch.cuda.synchronize()
            rc = _noalloc(lib, grid, U, got)
            assert rc == 0, f"call {call}: status {rc}"
            torch.cuda.synchronize()
            err = _rel(got, want)
            assert err <= TOL, f"call {call}: rel L2 {err:.3e}"


def test_noalloc_rejects_grids_beyond_the_fixed_scratch():
    import torch

    from ns3dperiodic_b200 import _lib

    lib = _lib.lib()
    grid = (128, 128, 128, 2 * np.pi, 2 * np.pi, 2 * np.pi)  # 1,064,960 points > 135,168
    shape = (128, 128, 65)
    U = [torch.zeros(shape, dtype=torch.complex128, device="cuda") for _ in range(3)]
    Q = [torch.full(shape, 7.0 + 0j, dtype=torch.complex128, device="cuda") for _ in range(3)]
    assert _noalloc(lib, grid, U, Q) == 1  # NS3D_ERR_BAD_ARG, nothing launched
    torch.cuda.synchronize()
    assert all(bool((q == 7.0).all()) for q in Q)
