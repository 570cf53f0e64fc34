"""A thin torch.autograd.Function over the C ABI, for gradient checks.

x = A(values)^{-1} b on a fixed sparsity pattern (one or many independent
systems). Forward: the mixed-precision solver (FP32 inner CG, FP64 residual
replacement) to a tight FP64 tolerance. Backward: the hand-written adjoint
(cmcg_cg_adjoint): one more solve A^T lambda = dL/dx with the same fused CG
(A symmetric), then dL/db = lambda and dL/dA_ij = -lambda_i x_j sampled on the
pattern by one kernel. Only the forward solution x is saved (checkpointed), no
iterate. The reference has no adjoint; this is not on its API.
"""
from __future__ import annotations

from typing import Optional

import numpy as np
import torch

from .solvers import ConjugateGradient, DiagonalPreconditioner
from .sparse import SparseMatrix, SparsityPattern


class SparseSolveOp:
    """Holds the pattern, an FP32 copy of the values for the inner solves, an
    FP64 copy for the residuals, and the solver."""

    def __init__(self, rows: int, row_ptr, col, row_off: Optional[np.ndarray] = None, tol: float = 1e-13,
                 max_outer: int = 200):
        self.pattern = SparsityPattern.csr(rows, rows, row_ptr, col)
        if row_off is not None:
            self.pattern.set_systems(row_off)
        self.A32 = SparseMatrix(self.pattern, dtype=torch.float32)
        self.A64 = SparseMatrix(self.pattern, dtype=torch.float64)
        self.cg = ConjugateGradient(self.A32, DiagonalPreconditioner)
        self.tol = tol
        self.max_outer = max_outer

    def set_values(self, values: torch.Tensor) -> None:
        """values: (nnz,) or (batches, nnz); a new batch count rebuilds the
        matrices and the solver on the same pattern."""
        v = values.detach().to(torch.float64).contiguous()
        batches = 1 if v.dim() == 1 else v.shape[0]
        if batches != self.A64.batches:
            self.A32 = SparseMatrix(self.pattern, dtype=torch.float32, batches=batches)
            self.A64 = SparseMatrix(self.pattern, dtype=torch.float64, batches=batches)
            self.cg = ConjugateGradient(self.A32, DiagonalPreconditioner)
        self.A64.setData(v)
        self.A32.setData(v)

    def solve(self, b: torch.Tensor) -> torch.Tensor:
        return self.cg.solve_refined(b.detach().to(torch.float64).contiguous(), outer=self.A64, outer_tol=self.tol,
                                     max_outer=self.max_outer)

    def adjoint(self, x: torch.Tensor, gx: torch.Tensor):
        return self.cg.adjoint(x, gx.to(torch.float64).contiguous(), outer=self.A64, outer_tol=self.tol,
                               max_outer=self.max_outer)


class SparseSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values: torch.Tensor, b: torch.Tensor, op: SparseSolveOp) -> torch.Tensor:
        op.set_values(values)
        x = op.solve(b)
        ctx.op = op
        ctx.values_shape = values.shape
        ctx.b_shape = b.shape
        # the op is shared and later forwards overwrite its values, so the
        # values of this call are saved and set again before its adjoint
        ctx.save_for_backward(x, values.detach().to(torch.float64))
        return x

    @staticmethod
    def backward(ctx, gx: torch.Tensor):
        x, values = ctx.saved_tensors
        ctx.op.set_values(values)
        gb, gA = ctx.op.adjoint(x, gx)
        gA = gA.reshape(-1, gA.shape[-1])
        if len(ctx.values_shape) < 2 or ctx.values_shape[0] == 1:
            # one value set broadcast over the batches of b: its gradient sums them
            gA = gA.sum(0)
        gb = gb.reshape(-1, x.shape[-1])
        if len(ctx.b_shape) < 2 or ctx.b_shape[0] == 1:
            gb = gb.sum(0)   # a one-batch b broadcast over batched values
        return gA.reshape(ctx.values_shape), gb.reshape(ctx.b_shape), None


def sparse_solve(values: torch.Tensor, b: torch.Tensor, op: SparseSolveOp) -> torch.Tensor:
    return SparseSolve.apply(values, b, op)
