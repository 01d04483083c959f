"""B200-native Position Based Fluids solver step (sm_100a CUDA behind a C ABI).

Drop-in for the solver interface of the reference (kernels/cudaPBF.h,
include/solver.h): see pbf_b200.solver.
"""
from ._lib import ExtParams, PBFError, SolverParameter, Stats, lib
from .solver import (BatchSolver, PBFSolver, Solver, cudaPBFSolve, default_ext, freeCUDASolverDataBuffer,
                     initCUDASolverDataBuffer, make_parameter)

__all__ = ["ExtParams", "PBFError", "SolverParameter", "Stats", "lib", "BatchSolver", "PBFSolver", "Solver",
           "cudaPBFSolve", "default_ext", "freeCUDASolverDataBuffer", "initCUDASolverDataBuffer", "make_parameter"]
