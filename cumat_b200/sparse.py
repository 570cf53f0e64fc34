"""Python mirror of cuMat's sparse / iterative-solver interface over the C ABI.

Names and argument meanings follow the reference so that code and tests read
like the reference's own (paths relative to the reference repository):

* ``SparsityPattern``  - cuMat/src/SparseMatrixBase.h:29-206 (CSR: ``JA`` row
  pointers, ``IA`` column indices; ELLPACK: ``indices`` column-major, -1 padding;
  ``assertValid()``)
* ``SparseMatrix``     - cuMat/src/SparseMatrix.h:48-414 (values ``[batch][nnz]``)
* ``A * x``            - operator*, cuMat/src/ProductOp.h:519-524
* ``dot`` / ``squaredNorm`` / ``norm`` - cuMat/src/ReductionOpsPlugin.inl:279-334
* ``ConjugateGradient`` with ``DiagonalPreconditioner`` (default) or
  ``IdentityPreconditioner`` - cuMat/src/ConjugateGradient.h:66-265,
  cuMat/src/IterativeSolverBase.h:10-135

Device vectors are torch tensors (torch provides device memory and the stream;
all arithmetic runs in this package's CUDA library). Vectors are shaped
``(n,)`` or ``(batches, n)``.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np
import torch

from . import _native as N

CSR = N.CSR
ELLPACK = N.ELLPACK
CSC = N.CSC
BSR = N.BSR

_TORCH_DT = {torch.float32: N.F32, torch.float64: N.F64, torch.bfloat16: N.BF16}
_NP_DT = {np.dtype(np.float32): N.F32, np.dtype(np.float64): N.F64}


def _vp(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr()) if isinstance(t, torch.Tensor) else C.c_void_p(t)


class Context:
    """Device + stream, like cuMat::Context (cuMat/src/Context.h:132-214).

    ``Context.current()`` binds the library to torch's current CUDA stream, so
    torch-produced inputs and library kernels are ordered on one stream.
    """

    _per_device: dict = {}

    LEGACY_DEFAULT_STREAM = 1  # cudaStreamLegacy

    def __init__(self, device: int = 0, stream: Optional[int] = None):
        """stream: a cudaStream_t value; None creates a private stream; 0 (torch's
        default stream) is taken as the legacy default stream."""
        self.device = device
        h = C.c_void_p()
        if stream == 0:
            stream = self.LEGACY_DEFAULT_STREAM
        N.call("cmcg_ctx_create", device, C.c_void_p(stream) if stream else None, C.byref(h))
        self.handle = h

    @classmethod
    def current(cls, device: Optional[int] = None) -> "Context":
        if device is None:
            device = torch.cuda.current_device()
        stream = torch.cuda.current_stream(device).cuda_stream
        key = (device, stream)
        ctx = cls._per_device.get(key)
        if ctx is None:
            ctx = cls(device, stream)
            cls._per_device[key] = ctx
        return ctx

    def synchronize(self) -> None:
        N.call("cmcg_ctx_synchronize", self.handle)

    def device_errors(self) -> int:
        """Synchronises and returns (and clears) the device error bits: 1 = a
        bulk-copy wait ran out, 2 = a grid barrier wait ran out."""
        f = C.c_int32(0)
        N.call("cmcg_ctx_device_errors", self.handle, C.byref(f))
        return int(f.value)

    @property
    def torch_device(self) -> torch.device:
        return torch.device("cuda", self.device)


class SparsityPattern:
    """Mirror of ``cuMat::SparsityPattern<CSR|CSC|ELLPACK>``; fill the fields,
    then ``assertValid()`` validates and uploads (the reference's assertValid
    only checks sizes; here malformed patterns raise ``CuMatError``). BSR
    (block CSR) stands for the reference's CSR pattern of block scalars."""

    def __init__(self, fmt: int = CSR):
        self.format = fmt
        self.rows = 0
        self.cols = 0
        self.nnz = 0            # CSR / CSC: stored entries; BSR: stored blocks
        self.IA = None          # CSR column indices / CSC row indices (nnz)
        self.JA = None          # CSR row pointers (rows + 1) / CSC column pointers (cols + 1)
        self.nnzPerRow = 0      # ELLPACK
        self.indices = None     # ELLPACK (rows, nnzPerRow), -1 = padding
        self.block = 1          # BSR block size; rows / cols count blocks
        self.handle = None
        self._ctx = None
        self.row_off = None

    # convenience constructors
    @classmethod
    def csr(cls, rows, cols, row_ptr, col_idx, ctx: Optional[Context] = None) -> "SparsityPattern":
        p = cls(CSR)
        p.rows, p.cols = int(rows), int(cols)
        p.JA = np.ascontiguousarray(row_ptr, dtype=np.int32)
        p.IA = np.ascontiguousarray(col_idx, dtype=np.int32)
        p.nnz = int(p.IA.size)
        p.assertValid(ctx)
        return p

    @classmethod
    def csc(cls, rows, cols, col_ptr, row_idx, ctx: Optional[Context] = None) -> "SparsityPattern":
        p = cls(CSC)
        p.rows, p.cols = int(rows), int(cols)
        p.JA = np.ascontiguousarray(col_ptr, dtype=np.int32)
        p.IA = np.ascontiguousarray(row_idx, dtype=np.int32)
        p.nnz = int(p.IA.size)
        p.assertValid(ctx)
        return p

    @classmethod
    def bsr(cls, block_rows, block_cols, block, row_ptr, col_idx, ctx: Optional[Context] = None) -> "SparsityPattern":
        """Block CSR: row_ptr / col_idx over blocks of block x block entries."""
        p = cls(BSR)
        p.rows, p.cols, p.block = int(block_rows), int(block_cols), int(block)
        p.JA = np.ascontiguousarray(row_ptr, dtype=np.int32)
        p.IA = np.ascontiguousarray(col_idx, dtype=np.int32)
        p.nnz = int(p.IA.size)
        p.assertValid(ctx)
        return p

    @classmethod
    def ell(cls, rows, cols, indices, ctx: Optional[Context] = None) -> "SparsityPattern":
        """indices: (rows, nnzPerRow) array (any memory order)."""
        p = cls(ELLPACK)
        ind = np.asarray(indices, dtype=np.int32)
        p.rows, p.cols = int(rows), int(cols)
        p.nnzPerRow = int(ind.shape[1])
        p.indices = ind
        p.assertValid(ctx)
        return p

    def assertValid(self, ctx: Optional[Context] = None) -> None:
        ctx = ctx or Context.current()
        self._ctx = ctx
        h = C.c_void_p()
        if self.format in (CSR, CSC, BSR):
            ja = np.ascontiguousarray(self.JA, dtype=np.int32)
            ia = np.ascontiguousarray(self.IA, dtype=np.int32)
            outer = self.cols if self.format == CSC else self.rows
            if ja.size != outer + 1 or ia.size != self.nnz:
                raise ValueError("SparsityPattern: JA must have outer size + 1 and IA nnz entries")
            iap = ia.ctypes.data_as(C.c_void_p) if ia.size else None
            if self.format == CSR:
                N.call("cmcg_pattern_create_csr", ctx.handle, self.rows, self.cols, self.nnz,
                       ja.ctypes.data_as(C.c_void_p), iap, 0, C.byref(h))
            elif self.format == CSC:
                N.call("cmcg_pattern_create_csc", ctx.handle, self.rows, self.cols, self.nnz,
                       ja.ctypes.data_as(C.c_void_p), iap, 0, C.byref(h))
            else:
                N.call("cmcg_pattern_create_bsr", ctx.handle, self.rows, self.cols, self.block, self.nnz,
                       ja.ctypes.data_as(C.c_void_p), iap, 0, C.byref(h))
        else:
            ind = np.asarray(self.indices, dtype=np.int32)
            if ind.shape != (self.rows, self.nnzPerRow):
                raise ValueError("SparsityPattern<ELLPACK>: indices must be rows x nnzPerRow")
            colmajor = np.ascontiguousarray(ind.T)  # [slot][row]
            N.call("cmcg_pattern_create_ell", ctx.handle, self.rows, self.cols, self.nnzPerRow,
                   colmajor.ctypes.data_as(C.c_void_p), 0, C.byref(h))
        self._release()
        self.handle = h

    def set_systems(self, row_off) -> None:
        """Declares independent diagonal blocks (packed batch of systems)."""
        ro = np.ascontiguousarray(row_off, dtype=np.int64)
        N.call("cmcg_pattern_set_systems", self.handle, ro.size - 1, ro.ctypes.data_as(C.c_void_p))
        self.row_off = ro

    def getNNZ(self) -> int:
        """Stored values per batch (BSR: block^2 per block)."""
        if self.format in (CSR, CSC):
            return self.nnz
        if self.format == BSR:
            return self.nnz * self.block * self.block
        return self.rows * self.nnzPerRow

    @property
    def scalar_rows(self) -> int:
        return self.rows * self.block if self.format == BSR else self.rows

    @property
    def scalar_cols(self) -> int:
        return self.cols * self.block if self.format == BSR else self.cols

    def download(self):
        """Device copy of the index arrays as given: (JA, IA) for CSR / CSC / BSR,
        (rows, width) indices for ELLPACK."""
        if self.format in (CSR, CSC, BSR):
            ja = np.empty((self.cols if self.format == CSC else self.rows) + 1, np.int32)
            ia = np.empty(max(self.nnz, 1), np.int32)
            N.call("cmcg_pattern_download", self.handle, ja.ctypes.data_as(C.c_void_p), ia.ctypes.data_as(C.c_void_p))
            return ja, ia[: self.nnz]
        out = np.empty((self.nnzPerRow, self.rows), np.int32)
        N.call("cmcg_pattern_download", self.handle, out.ctypes.data_as(C.c_void_p), None)
        return out.T.copy()

    def _release(self):
        if self.handle is not None:
            N.lib.cmcg_pattern_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self._release()
        except Exception:
            pass


class SparseMatrix:
    """Mirror of ``cuMat::SparseMatrix<Scalar, Batches, Flags>``: ``batches``
    value sets on one shared pattern."""

    def __init__(self, pattern: SparsityPattern, dtype=torch.float32, batches: int = 1):
        if pattern.handle is None:
            pattern.assertValid()
        self.pattern = pattern
        self.dtype = dtype
        self.batches = int(batches)
        h = C.c_void_p()
        N.call("cmcg_matrix_create", pattern.handle, _TORCH_DT[dtype], self.batches, C.byref(h))
        self.handle = h

    @property
    def rows(self) -> int:
        """Scalar rows (a BSR pattern's block rows times its block size)."""
        return self.pattern.scalar_rows

    @property
    def cols(self) -> int:
        return self.pattern.scalar_cols

    def getSparsityPattern(self) -> SparsityPattern:
        return self.pattern

    def setData(self, values) -> "SparseMatrix":
        """values: batch-major ``[batches][nnz]`` (CSR) or ``[batches][rows][width]``
        / ``[rows][width]`` (ELLPACK, converted to the column-major layout).
        numpy (host) or torch (host or device), F32 / F64 / BF16."""
        if self.pattern.format == ELLPACK:
            v = values if isinstance(values, torch.Tensor) else torch.as_tensor(np.asarray(values))
            if v.dim() == 2:
                v = v.unsqueeze(0)
            v = v.transpose(1, 2).contiguous()  # [b][slot][row]
            values = v
        if isinstance(values, torch.Tensor):
            t = values.contiguous()
            if t.dtype not in _TORCH_DT:
                t = t.to(torch.float64)
            if t.numel() != self.batches * self.pattern.getNNZ():
                raise ValueError("setData: expected batches * nnz values")
            N.call("cmcg_matrix_set_values", self.handle, _TORCH_DT[t.dtype], _vp(t), 1 if t.is_cuda else 0)
            if t.is_cuda:
                self.pattern._ctx.synchronize()
            return self
        a = np.ascontiguousarray(values)
        if a.dtype not in _NP_DT:
            a = a.astype(np.float64)
        if a.size != self.batches * self.pattern.getNNZ():
            raise ValueError("setData: expected batches * nnz values")
        N.call("cmcg_matrix_set_values", self.handle, _NP_DT[a.dtype], a.ctypes.data_as(C.c_void_p), 0)
        return self

    def getData(self) -> np.ndarray:
        """Values as stored (F32 / F64; BF16 returned as float32), batch-major."""
        n = self.batches * self.pattern.getNNZ()
        if self.dtype == torch.bfloat16:
            raw = np.empty(n, np.uint16)
            N.call("cmcg_matrix_get_values", self.handle, raw.ctypes.data_as(C.c_void_p))
            out = (raw.astype(np.uint32) << 16).view(np.float32)
        else:
            out = np.empty(n, np.float32 if self.dtype == torch.float32 else np.float64)
            N.call("cmcg_matrix_get_values", self.handle, out.ctypes.data_as(C.c_void_p))
        if self.pattern.format == ELLPACK:
            return out.reshape(self.batches, self.pattern.nnzPerRow, self.rows).transpose(0, 2, 1)
        if self.pattern.format == BSR:
            b = self.pattern.block
            return out.reshape(self.batches, self.pattern.nnz, b, b)
        return out.reshape(self.batches, self.pattern.nnz)

    def transposed_product(self, x: torch.Tensor, out: Optional[torch.Tensor] = None,
                           mode: int = N.ASSIGN) -> torch.Tensor:
        """out (mode)= A^T * x; x is (rows,) or (xb, rows)."""
        xb = 1 if x.dim() == 1 else x.shape[0]
        ob = max(self.batches, xb)
        if out is None:
            shape = (self.cols,) if (x.dim() == 1 and self.batches == 1) else (ob, self.cols)
            out = torch.empty(shape, dtype=x.dtype, device=x.device)
        x = x.contiguous()
        N.call("cmcg_spmv_transposed", self.handle, _TORCH_DT[x.dtype], _vp(x), xb, _vp(out), mode)
        return out

    def toDense(self, row_major: bool = True) -> torch.Tensor:
        """Dense copy (zeros off the pattern): (batches, rows, cols), on the device."""
        shape = (self.batches, self.rows, self.cols) if row_major else (self.batches, self.cols, self.rows)
        out = torch.empty(shape, dtype=self.dtype, device=self.pattern._ctx.torch_device)
        N.call("cmcg_matrix_to_dense", self.handle, _vp(out), 1 if row_major else 0)
        return out if row_major else out.transpose(1, 2)

    def setFromDense(self, dense: torch.Tensor) -> "SparseMatrix":
        """Takes the dense matrix's values at the pattern's entries (a sparse
        view of the dense matrix): dense (batches, rows, cols) or (rows, cols)."""
        d = dense.to(self.dtype)
        if d.dim() == 2:
            d = d.unsqueeze(0).expand(self.batches, -1, -1)
        d = d.contiguous()
        N.call("cmcg_matrix_from_dense", self.handle, _vp(d), 1)
        self.pattern._ctx.synchronize()
        return self

    def product(self, x: torch.Tensor, out: Optional[torch.Tensor] = None, mode: int = N.ASSIGN) -> torch.Tensor:
        """out (mode)= A * x; x is (cols,) or (xb, cols) float32/float64 on the device."""
        xb = 1 if x.dim() == 1 else x.shape[0]
        ob = max(self.batches, xb)
        if out is None:
            shape = (self.rows,) if (x.dim() == 1 and self.batches == 1) else (ob, self.rows)
            out = torch.empty(shape, dtype=x.dtype, device=x.device)
        x = x.contiguous()
        N.call("cmcg_spmv", self.handle, _TORCH_DT[x.dtype], _vp(x), xb, _vp(out), mode)
        return out

    def __mul__(self, x: torch.Tensor) -> torch.Tensor:
        return self.product(x)

    def __del__(self):
        try:
            if getattr(self, "handle", None) is not None:
                N.lib.cmcg_matrix_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


def dot(x: torch.Tensor, y: torch.Tensor) -> torch.Tensor:
    """Batched dot product: (n,) -> scalar tensor, (b, n) -> (b,)."""
    ctx = Context.current()
    xb = 1 if x.dim() == 1 else x.shape[0]
    yb = 1 if y.dim() == 1 else y.shape[0]
    n = x.shape[-1]
    ob = max(xb, yb)
    out = torch.empty(ob, dtype=x.dtype, device=x.device)
    N.call("cmcg_dot", ctx.handle, _TORCH_DT[x.dtype], n, _vp(x.contiguous()), xb, _vp(y.contiguous()), yb, _vp(out))
    return out[0] if (x.dim() == 1 and y.dim() == 1) else out


def squaredNorm(x: torch.Tensor) -> torch.Tensor:
    ctx = Context.current()
    b = 1 if x.dim() == 1 else x.shape[0]
    out = torch.empty(b, dtype=x.dtype, device=x.device)
    N.call("cmcg_squared_norm", ctx.handle, _TORCH_DT[x.dtype], x.shape[-1], _vp(x.contiguous()), b, _vp(out))
    return out[0] if x.dim() == 1 else out


def norm(x: torch.Tensor) -> torch.Tensor:
    return torch.sqrt(squaredNorm(x))


def linear_combination(coeffs, vectors, out: Optional[torch.Tensor] = None, mode: int = N.ASSIGN) -> torch.Tensor:
    """sum_t coeffs[t] * vectors[t] in one fused pass (up to 16 terms): the
    cwise expression ``v0 * f0 + v1 * f1 + ...`` of the reference. Vectors are
    (n,) or (b, n); one-batch vectors broadcast. mode ADD / SUB accumulates
    into ``out``."""
    vectors = [v.contiguous() for v in vectors]
    if len(vectors) != len(coeffs) or not 1 <= len(vectors) <= 16:
        raise ValueError("linear_combination: 1 to 16 (coefficient, vector) pairs")
    ctx = Context.current()
    n = vectors[0].shape[-1]
    vb = [1 if v.dim() == 1 else v.shape[0] for v in vectors]
    ob = max(vb)
    batched = any(v.dim() == 2 for v in vectors)
    if out is None:
        out = torch.empty((ob, n) if batched else (n,), dtype=vectors[0].dtype, device=vectors[0].device)
    cs = (C.c_double * len(coeffs))(*[float(c) for c in coeffs])
    ptrs = (C.c_void_p * len(vectors))(*[v.data_ptr() for v in vectors])
    bs = (C.c_int32 * len(vectors))(*vb)
    N.call("cmcg_lincomb", ctx.handle, _TORCH_DT[vectors[0].dtype], n, len(vectors), cs, ptrs, bs, _vp(out), ob,
           int(mode))
    return out


def sddmm(A: SparseMatrix, u: torch.Tensor, v: torch.Tensor, alpha: float = 1.0) -> torch.Tensor:
    """alpha * u v^T sampled on A's pattern, in A's value layout ([batch][nnz])."""
    ub = 1 if u.dim() == 1 else u.shape[0]
    vb = 1 if v.dim() == 1 else v.shape[0]
    ob = max(ub, vb)
    out = torch.empty((ob, A.pattern.getNNZ()), dtype=u.dtype, device=u.device)
    N.call("cmcg_sddmm", A.handle, _TORCH_DT[u.dtype], float(alpha), _vp(u.contiguous()), ub, _vp(v.contiguous()), vb,
           _vp(out), ob)
    return out


_REDUCE_OPS = {"sum": N.REDUCE_SUM, "prod": N.REDUCE_PROD, "min": N.REDUCE_MIN, "max": N.REDUCE_MAX}
_AXES = {"rows": N.AXIS_ROW, "cols": N.AXIS_COLUMN, "batches": N.AXIS_BATCH}


def reduce(x: torch.Tensor, op: str = "sum", axes=("rows",)) -> torch.Tensor:
    """Reduction of a dense batched matrix along any set of axes, like the
    reference's ``sum<ReductionAxis::Row | ...>()`` / ``prod`` / ``minCoeff`` /
    ``maxCoeff``. ``x`` is (batches, cols, rows) in memory order (rows fastest,
    the reference's ColumnMajor; a 2-D tensor is one batch); ``axes`` names the
    reduced ones. Returns the kept axes in the same order, reduced axes kept
    with size 1."""
    if x.dim() == 2:
        x = x.unsqueeze(0)
    B, Cc, R = x.shape
    mask = 0
    for a in axes:
        mask |= _AXES[a]
    out = torch.empty((1 if mask & N.AXIS_BATCH else B, 1 if mask & N.AXIS_COLUMN else Cc,
                       1 if mask & N.AXIS_ROW else R), dtype=x.dtype, device=x.device)
    N.call("cmcg_reduce", Context.current().handle, _TORCH_DT[x.dtype], _REDUCE_OPS[op], R, Cc, B, mask,
           _vp(x.contiguous()), _vp(out))
    return out


_log_keep = []


def set_log_callback(fn, max_level: int = 1) -> None:
    """Routes the library's log messages (level 0 errors, 1 decisions such as
    tuned kernels and FP32 fallbacks, 2 details of every solve) to
    ``fn(level, message)``; ``None`` removes the callback."""
    if fn is None:
        N.call("cmcg_set_log_callback", None, 0, None)
        _log_keep.clear()
        return
    proto = C.CFUNCTYPE(None, C.c_int32, C.c_char_p, C.c_void_p)
    cb = proto(lambda level, msg, user: fn(int(level), msg.decode(errors="replace")))
    _log_keep[:] = [cb]
    N.call("cmcg_set_log_callback", C.cast(cb, C.c_void_p), int(max_level), None)
