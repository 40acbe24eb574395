"""B200-native HOPS trajectory hot path with the MesoHOPS drop-in surface.

Public API:
  HopsTrajectory  -- drop-in for mesohops.trajectory.hops_trajectory.HopsTrajectory
  HopsEnsemble    -- B trajectories sharing one hierarchy, batched on one GPU
  DyadicTrajectory -- drop-in for mesohops.trajectory.hops_dyadic.DyadicTrajectory
  bcf_exp, bcf_convert_dl_to_exp -- bath helpers for system dictionaries
The CUDA library is mesohops_b200/lib/libhops_b200.so (C ABI in
include/hops_b200.h); build it with ``python -m mesohops_b200.build``.
"""
from .bath import bcf_convert_dl_to_exp, bcf_exp
from .constants import hbar, kB, precision
from .exceptions import AuxError, LockedException, TrajectoryError, UnsupportedRequest

__version__ = "0.1.0"


def __getattr__(name):
    # torch-dependent modules load lazily so that `import mesohops_b200` stays cheap
    if name == "HopsTrajectory":
        from .trajectory import HopsTrajectory
        return HopsTrajectory
    if name == "HopsEnsemble":
        from .ensemble import HopsEnsemble
        return HopsEnsemble
    if name == "DyadicTrajectory":
        from .dyadic import DyadicTrajectory
        return DyadicTrajectory
    raise AttributeError(name)
