"""metal4foam_b200 -- B200-native (sm_100a) Krylov hot path of the metal4Foam
OpenFOAM plugin: the cudaPCG / cudaPBiCGStab lduMatrix solvers over the C ABI
of libcudafoam.so (include/cudafoam.h)."""
from . import mesh
from ._lib import Context, CudaFoamError, default_options, load
from .solver import (FatalError, cudaFoamSolver, cudaPBiCGStab, cudaPCG, lduAddressing,
                     lduMatrix, solverPerformance)

__all__ = ["mesh", "Context", "CudaFoamError", "default_options", "load", "FatalError",
           "cudaFoamSolver", "cudaPCG", "cudaPBiCGStab", "lduAddressing", "lduMatrix",
           "solverPerformance"]
