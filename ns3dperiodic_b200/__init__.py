"""B200 (sm_100a) pseudo-spectral Navier-Stokes RK3 path, a drop-in for the
time-stepping / Jacobian / Krylov entry points of NS3DPeriodic.

The compute path is the CUDA library libns3d_b200.so (C ABI in
include/ns3d.h); :class:`Solver` (time stepping), :class:`Ensemble` (many instances of one
grid stepped together) and :class:`Krylov` (Arnoldi / implicit restart) are
the Python host mirrors over it.
"""
from ._lib import Ns3dError, Ns3dLibraryError, LIB_PATH  # noqa: F401
from .solver import (Ensemble, Server, Solver, TimeSeries, request_steps,  # noqa: F401
                     supported_extent)
from .krylov import Krylov, qr_shifts, select_shifts  # noqa: F401

__all__ = ["Solver", "Ensemble", "Server", "TimeSeries", "request_steps", "supported_extent", "Krylov", "qr_shifts", "select_shifts", "Ns3dError",
           "Ns3dLibraryError", "LIB_PATH"]
