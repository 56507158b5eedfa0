"""Device checkpoints through the C ABI (ns3d_save/load_control_fourier,
ns3d_save/load_control_file): the files carry the device state exactly
(%.16le round trips FP64), a coarser Fourier file is up-sampled as the host
reader (pinned against the reference's read_control_fourier on the CPU) does,
and the physical file holds the inverse transform of the state."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t

    if not t.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return t


def _rand_spectral(torch, S, seed):
    g = torch.Generator(device="cpu").manual_seed(seed)
    shape = (S.Nx, S.Ny, S.Nz)
    return [S.fftn(torch.randn(shape, generator=g, dtype=torch.float64).cuda()) for _ in range(3)]


@pytest.mark.parametrize("shape", [(16, 16, 16), (32, 16, 24), (64, 64, 64)])
def test_fourier_checkpoint_round_trip_is_exact(torch, tmp_path, shape):
    from ns3dperiodic_b200 import Solver
    from ns3dperiodic_b200 import solver as SM

    S = Solver(*shape)
    U = _rand_spectral(torch, S, sum(shape))
    path = tmp_path / "control_file_Fourier.dat"
    S.save_control_fourier(path, U)
    host, ext = SM.read_control_fourier(path, *shape)
    assert ext == (shape[0], shape[1], shape[2] // 2 + 1)
    for a, b in zip(host, U):
        np.testing.assert_array_equal(a, b.cpu().numpy())
    V = S.load_control_fourier(path)
    for a, b in zip(V, U):
        assert torch.equal(a, b)
    S.close()


def test_coarse_fourier_checkpoint_is_upsampled_on_load(torch, tmp_path):
    from ns3dperiodic_b200 import Solver
    from ns3dperiodic_b200 import solver as SM

    coarse = Solver(16, 16, 16)
    U = _rand_spectral(torch, coarse, 7)
    path = tmp_path / "control_file_Fourier.dat"
    coarse.save_control_fourier(path, U)
    fine = Solver(32, 32, 32)
    V = fine.load_control_fourier(path)
    host, ext = SM.read_control_fourier(path, 32, 32, 32)
    assert ext == (16, 16, 9)
    for a, b in zip(V, host):
        np.testing.assert_array_equal(a.cpu().numpy(), b)
    # the reference's integer scale: (32*32*33) // (16*16*17) = 7
    np.testing.assert_array_equal(V[0][1, 2, 3].cpu().numpy(), 7 * U[0][1, 2, 3].cpu().numpy())
    np.testing.assert_array_equal(V[1][-3, -5, 8].cpu().numpy(), 7 * U[1][-3, -5, 8].cpu().numpy())
    coarse.close()
    fine.close()


@pytest.mark.parametrize("shape", [(16, 16, 16), (24, 32, 16)])
def test_physical_checkpoint_holds_the_velocity(torch, tmp_path, shape):
    from ns3dperiodic_b200 import Solver
    from ns3dperiodic_b200 import solver as SM

    S = Solver(*shape)
    U = _rand_spectral(torch, S, 11)
    path = tmp_path / "control_file.dat"
    S.save_control_file(path, U)
    u = SM.read_control_file(path, *shape)
    for a, b in zip(u, U):
        np.testing.assert_array_equal(a, S.ifftn(b).cpu().numpy())
    V = S.load_control_file(path)
    for a, b in zip(V, u):
        assert torch.equal(a, S.fftn(torch.as_tensor(b).cuda()))
    S.close()


def test_mismatched_checkpoint_is_an_error(torch, tmp_path):
    from ns3dperiodic_b200 import Ns3dError, Solver

    big = Solver(32, 32, 32)
    big.save_control_fourier(tmp_path / "big.dat", _rand_spectral(torch, big, 3))
    small = Solver(16, 16, 16)
    with pytest.raises(Ns3dError):
        small.load_control_fourier(tmp_path / "big.dat")
    with pytest.raises(Ns3dError):
        small.load_control_file(tmp_path / "big.dat")
    big.close()
    small.close()
