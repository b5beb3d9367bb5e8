"""nekwave_b200: B200-native (sm_100a) DG-SEM Maxwell RHS + LSRK45 step of NekWave.

The compute path is libnwb.so (CUDA kernels + C ABI, include/nwb.h); this
package mirrors the reference's DgSolver/Mesh interface on top of it.
"""
from .dg_solver import DgSolver, StateVector  # noqa: F401
from .mesh import Mesh  # noqa: F401

__all__ = ["DgSolver", "Mesh", "StateVector"]
