"""The bounded device waits of the tensor-copy passes give up instead of
hanging: ns3d_selftest_bounded_wait runs one CTA that waits on an mbarrier
phase nothing completes; the wait must give up after about 0.1 s with the
timeout code on its device flag, and the device must stay usable (a solver
step right after it matches the same step before it bit for bit)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t

    if not t.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return t


def test_wait_gives_up_and_the_device_stays_usable(torch):
    from ns3dperiodic_b200 import Solver
    from ns3dperiodic_b200 import workload as W
    from ns3dperiodic_b200._lib import lib

    N, Re = 32, 200.0
    U0, F = W.kolmogorov_state(N, Re, 2, rel_amp=0.05)
    dt = W.kolmogorov_dt(N, Re)
    with Solver(N, N, N) as S:
        S.set_forcing(S.to_device(F))
        before = [u.cpu().numpy() for u in S.rk3_ssp(S.to_device(U0), dt, Re, nsteps=2)]
        secs = ctypes.c_double(-1.0)
        assert lib().ns3d_selftest_bounded_wait(ctypes.byref(secs)) == 0
        assert 0.05 < secs.value < 5.0, secs.value
        after = [u.cpu().numpy() for u in S.rk3_ssp(S.to_device(U0), dt, Re, nsteps=2)]
        S.synchronize()
    assert all(np.array_equal(a, b) for a, b in zip(after, before))
