"""B200 implementation of ns3d_cpp's RHS + RK3 time-step loop (periodic box).

The compute path is ``libns3d_b200.so`` (hand-written sm_100a CUDA behind the C
ABI of ``include/ns3d_gpu.h``); this package is the host-side mirror of the
reference's solver interface plus initial-condition generators.
"""
from .solver import (NS3DError, Solver, SolverParams, read_solver_params_from_file)  # noqa: F401
from . import initial  # noqa: F401
