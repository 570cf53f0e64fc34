"""ConjugateGradient and preconditioners (mirror of cuMat/src/ConjugateGradient.h:66-265
and cuMat/src/IterativeSolverBase.h:10-135) over the C ABI."""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np
import torch

from . import _native as N
from .sparse import SparseMatrix, _TORCH_DT, _vp


class DiagonalPreconditioner:
    """Jacobi: 1 / a_ii per batch, 1 where a_ii is zero or absent
    (reference DiagonalPreconditioner + cwiseInverseCheck)."""
    code = N.PRECOND_JACOBI


class IdentityPreconditioner:
    code = N.PRECOND_IDENTITY


class ConjugateGradient:
    """``ConjugateGradient(A).setTolerance(t).solve(b)``; ``iterations()`` and
    ``error()`` report the largest value over all systems of the last solve.

    Deviation from the reference, by design: each (batch, system) stops on its
    own convergence instead of iterating until every batch has converged, and a
    breakdown or non-finite scalar stops that system with a status
    (``system_stats``) instead of propagating NaNs.
    """

    def __init__(self, A: SparseMatrix, preconditioner=DiagonalPreconditioner):
        self.A = A
        self.precond = preconditioner
        h = C.c_void_p()
        N.call("cmcg_cg_create", A.handle, preconditioner.code, C.byref(h))
        self.handle = h
        self._last_batches = 0

    # -- settings (IterativeSolverBase.h:54-95) --
    def setTolerance(self, tol: float) -> "ConjugateGradient":
        N.call("cmcg_cg_set_tolerance", self.handle, float(tol))
        return self

    def setMaxIterations(self, max_iter: int) -> "ConjugateGradient":
        N.call("cmcg_cg_set_max_iterations", self.handle, int(max_iter))
        return self

    def set_path(self, path: int) -> "ConjugateGradient":
        N.call("cmcg_cg_set_path", self.handle, int(path))
        return self

    def set_refinement(self, method: int = N.REFINE_RELIABLE, delta: float = 0.0) -> "ConjugateGradient":
        """Mixed-precision method of solve_refined: reliable updates (default) or restarts;
        delta 0 picks the replacement threshold by the inner value type (0.01 FP32, 0.1 BF16)."""
        N.call("cmcg_cg_set_refinement", self.handle, int(method), float(delta))
        return self

    def tolerance(self) -> float:
        t, m = C.c_double(), C.c_int64()
        N.call("cmcg_cg_get_settings", self.handle, C.byref(t), C.byref(m))
        return t.value

    def maxIterations(self) -> int:
        t, m = C.c_double(), C.c_int64()
        N.call("cmcg_cg_get_settings", self.handle, C.byref(t), C.byref(m))
        return m.value

    # -- solves --
    def solve(self, b: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        return self.solveWithGuess(b, None, out)

    def solveWithGuess(self, b: torch.Tensor, guess: Optional[torch.Tensor], out: Optional[torch.Tensor] = None) -> torch.Tensor:
        bb = 1 if b.dim() == 1 else b.shape[0]
        ob = max(self.A.batches, bb)
        if out is None:
            shape = (self.A.rows,) if (b.dim() == 1 and self.A.batches == 1) else (ob, self.A.rows)
            out = torch.empty(shape, dtype=b.dtype, device=b.device)
        g = None
        if guess is not None:
            g = guess.expand(ob, self.A.rows).contiguous() if guess.dim() == 1 and ob > 1 else guess.contiguous()
        N.call("cmcg_cg_solve", self.handle, _TORCH_DT[b.dtype], _vp(b.contiguous()), bb,
               _vp(g) if g is not None else None, _vp(out))
        self._last_batches = ob
        return out

    def solve_host(self, b: np.ndarray, batches: int = 1, guess: Optional[np.ndarray] = None) -> np.ndarray:
        """Host buffers in and out (upload, solve, download inside the library)."""
        b = np.ascontiguousarray(b)
        dt = N.F32 if b.dtype == np.float32 else N.F64
        ob = max(self.A.batches, batches)
        x = np.empty((ob, self.A.rows), dtype=b.dtype)
        N.call("cmcg_cg_solve_host", self.handle, dt, b.ctypes.data_as(C.c_void_p), batches,
               np.ascontiguousarray(guess, dtype=b.dtype).ctypes.data_as(C.c_void_p) if guess is not None else None,
               x.ctypes.data_as(C.c_void_p))
        self._last_batches = ob
        return x

    def solve_refined(self, b: torch.Tensor, outer: Optional[SparseMatrix] = None, outer_tol: float = 1e-10,
                      max_outer: int = 20, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        """Mixed precision: FP32 (F32 / BF16 values) inner CG at this solver's
        tolerance, FP64 residual / update / norms with ``outer``'s values (F32 or
        F64; default this solver's matrix) until |b - A x| < outer_tol |b|."""
        assert b.dtype == torch.float64
        bb = 1 if b.dim() == 1 else b.shape[0]
        ob = max(self.A.batches, bb)
        if out is None:
            shape = (self.A.rows,) if (b.dim() == 1 and self.A.batches == 1) else (ob, self.A.rows)
            out = torch.empty(shape, dtype=torch.float64, device=b.device)
        N.call("cmcg_cg_solve_refined", self.handle, outer.handle if outer is not None else None,
               _vp(b.contiguous()), bb, _vp(out), float(outer_tol), int(max_outer))
        self._last_batches = ob
        return out

    def adjoint(self, x: torch.Tensor, gx: torch.Tensor, outer: Optional[SparseMatrix] = None,
                outer_tol: float = 1e-12, max_outer: int = 30, want_gA: bool = True):
        """Given the forward solution x and dL/dx, returns (dL/db, dL/dA on the
        pattern as [batch][nnz]) by one adjoint solve + one sampled outer product."""
        batches = 1 if x.dim() == 1 else x.shape[0]
        gb = torch.empty_like(x, dtype=torch.float64)
        gA = torch.empty((max(self.A.batches, batches), self.A.pattern.getNNZ()), dtype=torch.float64,
                         device=x.device) if want_gA else None
        N.call("cmcg_cg_adjoint", self.handle, outer.handle if outer is not None else None, _vp(x.contiguous()),
               _vp(gx.contiguous()), batches, _vp(gb), _vp(gA) if gA is not None else None, float(outer_tol),
               int(max_outer))
        self._last_batches = max(self.A.batches, batches)
        return gb, gA

    # -- results (IterativeSolverBase.h:97-111) --
    def iterations(self) -> int:
        v = C.c_int64()
        N.call("cmcg_cg_iterations", self.handle, C.byref(v))
        return v.value

    def error(self) -> float:
        v = C.c_double()
        N.call("cmcg_cg_error", self.handle, C.byref(v))
        return v.value

    def system_stats(self, n_inst: Optional[int] = None):
        """Per (batch, system) arrays: iterations, error, status, refinement steps,
        and (refined solves with BF16 values) whether the system was solved again
        with FP32 values."""
        if n_inst is None:
            ns = 1 if self.A.pattern.row_off is None else self.A.pattern.row_off.size - 1
            n_inst = self._last_batches * ns
        it = np.empty(n_inst, np.int32)
        err = np.empty(n_inst, np.float64)
        st = np.empty(n_inst, np.int32)
        ou = np.empty(n_inst, np.int32)
        N.call("cmcg_cg_system_stats", self.handle, it.ctypes.data_as(C.c_void_p), err.ctypes.data_as(C.c_void_p),
               st.ctypes.data_as(C.c_void_p), ou.ctypes.data_as(C.c_void_p))
        fb = np.zeros(n_inst, np.int32)
        N.call("cmcg_cg_fallbacks", self.handle, fb.ctypes.data_as(C.c_void_p), None)
        return {"iterations": it, "error": err, "status": st, "outer": ou, "fallback": fb}

    def __del__(self):
        try:
            if getattr(self, "handle", None) is not None:
                N.lib.cmcg_cg_destroy(self.handle)
                self.handle = None
        except Exception:
            pass
