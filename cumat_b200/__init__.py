"""cumat_b200 — sm_100a batched sparse conjugate-gradient path of cuMat.

The compute path is the CUDA library lib/libcumat_cg.so behind the C ABI in
include/cumat_cg.h; this package is its Python mirror of cuMat's interface.
Importing fails if the library has not been built (no CPU fallback).
"""
from . import _native
from ._native import CuMatError, launch_count
from .sparse import (CSR, ELLPACK, Context, SparseMatrix, SparsityPattern, dot, linear_combination, norm, sddmm,
                     squaredNorm)
from .solvers import ConjugateGradient, DiagonalPreconditioner, IdentityPreconditioner

__all__ = [
    "CSR", "ELLPACK", "Context", "SparseMatrix", "SparsityPattern", "dot", "linear_combination", "norm", "squaredNorm",
    "sddmm",
    "ConjugateGradient", "DiagonalPreconditioner", "IdentityPreconditioner", "CuMatError", "launch_count",
]
