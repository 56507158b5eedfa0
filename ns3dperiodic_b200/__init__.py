"""B200 (sm_100a) pseudo-spectral Navier-Stokes RK3 path, a drop-in for the
time-stepping / Jacobian / Krylov-matvec entry points of NS3DPeriodic.

The compute path is the CUDA library libns3d_b200.so (C ABI in
include/ns3d.h); :class:`Solver` is the Python host mirror over it.
"""
from ._lib import Ns3dError, Ns3dLibraryError, LIB_PATH  # noqa: F401
from .solver import Solver, supported_extent  # noqa: F401

__all__ = ["Solver", "supported_extent", "Ns3dError", "Ns3dLibraryError", "LIB_PATH"]
