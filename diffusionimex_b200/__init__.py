"""B200-native SPB 6+1-equation two-phase IMEX solver.

The hot path -- the SPB6_PC_IMEX stage loop of the diffusionIMEX reference --
runs as hand-written sm_100a CUDA kernels behind the C ABI in include/spb6g.h;
this package holds the kernels (csrc/), the build recipe (build.py), the
ctypes host layer (solver.py) and the initial-data generators (cases.py).
"""
from . import cases
from .solver import BatchSolver, Solver, SolverError, format_profile, library, run_main

__all__ = ["BatchSolver", "Solver", "SolverError", "cases", "format_profile", "library", "run_main"]
