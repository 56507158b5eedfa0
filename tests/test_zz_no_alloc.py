"""The allocation-free nonlinear term, ns3d_convolution_noalloc.

It exists for callers that cannot allocate device memory on the call path:
programs that reserve all device memory up front for their own pool, callers
that keep no handle between calls, and code that cannot take the
synchronisation cudaMalloc/cudaFree may cost.  It must give the same result as
the handle-based ns3d_convolution while working only in the scratch array
compiled into the library.

This file is collected last on purpose (a failure here stops an -x run only
after every other test has run).  It passes on its own in a fresh process as
well, and one case runs in a child process that never creates a handle, so
the entry point's first-call set-up runs there with no other library state.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative L2, the tolerance of the other GPU parity tests
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


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


def test_noalloc_alternating_grids_and_a_side_stream():
    """Grids and boxes that change from call to call reload the cached tables;
    every call, on a non-default stream, equals ns3d_convolution of a handle
    for the same grid."""
    import torch

    from ns3dperiodic_b200 import Solver, _lib

    lib = _lib.lib()
    grids = [(32, 24, 48, 2 * np.pi, 3.0, 5.0), (16, 16, 16, 2 * np.pi, 2 * np.pi, 2 * np.pi),
             (32, 24, 48, 2 * np.pi, 3.0, 5.0), (32, 24, 48, 1.0, 2.0, 3.0),
             (64, 32, 16, 2 * np.pi, np.pi, 2 * np.pi)]
    side = torch.cuda.Stream()
    for call, grid in enumerate(grids):
        with Solver(*grid) as S:
            U = S.to_device(_field(S.shape, 10 + call))
            want = S.calculate_convolution_2p3(U)
            got = [torch.full(S.shape, complex(np.nan, np.nan), dtype=torch.complex128,
                              device=S.device) for _ in range(3)]
            torch.cuda.synchronize()
            rc = _noalloc(lib, grid, U, got, stream=side.cuda_stream)
            assert rc == 0, f"call {call} {grid[:3]}: status {rc}"
            side.synchronize()
            err = _rel(got, want)
            assert err <= TOL, f"call {call} {grid}: rel L2 {err:.3e}"


_CHILD = r"""
import ctypes, sys
import numpy as np
import torch
sys.path.insert(0, {root!r})
from oracle import ns3d_oracle as O
from ns3dperiodic_b200 import _lib
from tests.test_zz_no_alloc import _field, _noalloc

lib = _lib.lib()
torch.cuda.init()
errs = []
for seed, grid in enumerate([(16, 24, 32, 2 * np.pi, 3.0, 5.0), (16, 24, 32, 2 * np.pi, 3.0, 5.0)]):
    Nx, Ny, Nz = grid[:3]
    g = O.Grid(Nx, Ny, Nz, *grid[3:])
    Uh = _field(g.shape_c, 30 + seed)
    U = [torch.from_numpy(u).cuda() for u in Uh]
    Q = [torch.full(g.shape_c, complex(np.nan, np.nan), dtype=torch.complex128, device="cuda")
         for _ in range(3)]
    torch.cuda.synchronize()
    rc = _noalloc(lib, grid, U, Q)
    torch.cuda.synchronize()
    if rc != 0:
        print("status", rc)
        sys.exit(2)
    errs.append(O.rel_l2([q.cpu().numpy() for q in Q], O.convolution(g, Uh)))
print("errs", *errs)
sys.exit(0 if all(e <= {tol!r} for e in errs) else 1)
"""


def test_noalloc_first_call_in_a_process_without_a_handle():
    """A fresh process whose first library call is the allocation-free entry
    point (no ns3d_create before it): two calls against the CPU oracle."""
    code = _CHILD.format(root=ROOT, tol=TOL)
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr


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
