"""Plain 3-D transforms (FFTN_Device / iFFTN_Device) through the C ABI against
cuFFT (torch.fft runs cuFFT on the GPU), the reference's own cuFFT call on a
non-Hermitian spectrum (golden vectors) and the oracle.  Tolerance: relative
L2 <= 1e-13 (FP64 transforms agree to a few ulp times log N).
"""
import numpy as np
import pytest

from oracle import ns3d_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-13

GRIDS = [(16, 16, 16), (32, 48, 24), (64, 64, 64), (8, 96, 16), (128, 128, 128),
         (24, 16, 384), (256, 8, 8), (48, 512, 8), (256, 256, 256)]


@pytest.fixture(scope="module")
def torch():
    import torch as t

    if not t.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return t


def _rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.mark.parametrize("shape", GRIDS)
def test_r2c_and_c2r_match_cufft(torch, shape):
    from ns3dperiodic_b200 import Solver

    Nx, Ny, Nz = shape
    S = Solver(Nx, Ny, Nz)
    g = torch.Generator(device="cpu").manual_seed(Nx * 7 + Ny * 3 + Nz)
    x = torch.randn(shape, generator=g, dtype=torch.float64).cuda()
    X = S.fftn(x)
    Xref = torch.fft.rfftn(x).contiguous()  # cuFFT D2Z, unnormalised
    assert _rel(X.cpu().numpy(), Xref.cpu().numpy()) < TOL
    y = S.ifftn(Xref)
    yref = torch.fft.irfftn(Xref, s=shape)  # cuFFT Z2D with the 1/N scale
    assert _rel(y.cpu().numpy(), yref.cpu().numpy()) < TOL
    assert _rel(y.cpu().numpy(), x.cpu().numpy()) < TOL
    S.close()


def test_c2r_keeps_input_and_matches_reference_on_non_hermitian_planes(torch, golden):
    """The reference's Nyquist convention makes the kz = 0 / Nz/2 planes
    non-Hermitian; cuFFT's Z2D (run by the reference build) uses only their
    Hermitian part."""
    from ns3dperiodic_b200 import Solver

    for case in ("iso16", "aniso16x8x24"):
        d = golden[case]
        S = Solver(int(d["Nx"]), int(d["Ny"]), int(d["Nz"]), float(d["Lx"]), float(d["Ly"]),
                   float(d["Lz"]))
        Xn = torch.as_tensor(d["X_nonherm"]).cuda()
        keep = Xn.clone()
        y = S.ifftn(Xn)
        assert torch.equal(Xn, keep)
        assert _rel(y.cpu().numpy(), d["c2r_nonherm"]) < TOL
        S.close()


def test_transforms_vs_oracle_anisotropic_box(torch):
    from ns3dperiodic_b200 import Solver

    g = O.Grid(48, 32, 64, 3.0, 2.0, 5.0)
    S = Solver(48, 32, 64, 3.0, 2.0, 5.0)
    rng = np.random.default_rng(3)
    x = rng.standard_normal((48, 32, 64))
    X = S.fftn(torch.as_tensor(x).cuda())
    assert _rel(X.cpu().numpy(), O.r2c(g, x)) < TOL
    Y = rng.standard_normal(g.shape_c) + 1j * rng.standard_normal(g.shape_c)
    y = S.ifftn(torch.as_tensor(Y).cuda())
    assert _rel(y.cpu().numpy(), O.c2r(g, Y)) < TOL
    S.close()


def test_round_trip_512_cubed(torch):
    """Size-independent property at the largest grid: C2R(R2C(x)) = x."""
    from ns3dperiodic_b200 import Solver

    S = Solver(512, 512, 512)
    x = torch.randn((512, 512, 512), dtype=torch.float64, device="cuda")
    X = S.fftn(x)
    y = S.ifftn(X)
    err = (torch.linalg.vector_norm(y - x) / torch.linalg.vector_norm(x)).item()
    assert err < 1e-14
    # Parseval: sum x^2 = (1/N) sum over the full spectrum |X|^2
    w = torch.full((X.shape[-1],), 2.0, dtype=torch.float64, device="cuda")
    w[0] = 1.0
    w[-1] = 1.0
    lhs = torch.sum(x * x).item()
    rhs = (torch.sum((X.real ** 2 + X.imag ** 2) * w) / 512 ** 3).item()
    assert abs(lhs / rhs - 1.0) < 1e-12
    del X, y
    S.close()
