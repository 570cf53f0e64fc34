"""cumat_b200 — sm_100a batched sparse conjugate-gradient path of cuMat.

The compute path is the CUDA library lib/libcumat_cg.so behind the C ABI in
include/cumat_cg.h; this package is its Python mirror of cuMat's interface.
Importing fails if the library has not been built (no CPU fallback).
"""
from . import _native
from ._native import CuMatError, launch_count
from .sparse import (BSR, CSC, CSR, ELLPACK, Context, SparseMatrix, SparsityPattern, dot, linear_combination, norm,
                     reduce, sddmm, set_log_callback, squaredNorm)
from .solvers import ConjugateGradient, DiagonalPreconditioner, IdentityPreconditioner

__all__ = [
    "CSR", "CSC", "BSR", "ELLPACK", "Context", "SparseMatrix", "SparsityPattern", "dot", "linear_combination", "norm",
    "squaredNorm", "sddmm", "reduce", "set_log_callback",
    "ConjugateGradient", "DiagonalPreconditioner", "IdentityPreconditioner", "CuMatError", "launch_count",
]
