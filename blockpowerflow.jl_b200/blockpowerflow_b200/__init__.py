"""BlockPowerFlow-B200: the multi-RHS sparse solve path of exanauts/BlockPowerFlow.jl on B200.

Python mirror of the reference's Julia API (module BlockPowerFlow, src/BlockPowerFlow.jl):
block_gmres, block_bicgstab, ilu0, ic0, ldiv!, CUSOLVERRF; plus the batched solve of many
independent systems in one graph launch (BatchPlan).  Every call runs in libbpf.so
(hand-written sm_100a kernels); there is no CPU fallback.
"""
from . import cusolverrf as CUSOLVERRF
from . import grid
from .batch import BatchPlan, BatchStats, autotune
from ._lib import (BPFError, DimensionMismatch, SingularException, exported_symbols,
                   kernel_launches)
from .krylov import (BlockBicgstabSolver, BlockGMRESSolver, BlockGMRESStats, SimpleStats, block_bicgstab,
                     block_bicgstab_, block_gmres, block_gmres_, warm_start_)
from .precond import NVIDIA_IC0, NVIDIA_ILU0, BlockJacobiPreconditioner, ic0, ilu0, ldiv_, mul_
from .sparse import CuSparseMatrixCSR, colmajor, empty_colmajor, householder, mul

ldiv = ldiv_

__all__ = [
    "block_gmres", "block_bicgstab", "BlockGMRESStats", "SimpleStats", "ilu0", "ic0", "ldiv_",
    "ldiv", "NVIDIA_ILU0", "NVIDIA_IC0", "CuSparseMatrixCSR", "mul", "householder", "colmajor",
    "empty_colmajor", "BPFError", "DimensionMismatch", "SingularException", "grid",
    "exported_symbols", "kernel_launches", "CUSOLVERRF", "BatchPlan", "BatchStats", "autotune",
    "BlockJacobiPreconditioner", "mul_", "BlockGMRESSolver", "BlockBicgstabSolver", "block_gmres_",
    "block_bicgstab_", "warm_start_",
]
