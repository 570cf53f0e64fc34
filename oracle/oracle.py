"""CPU ORACLE — test infrastructure only (see oracle/__init__.py).

numpy front end of two libraries built by oracle/Makefile:
  liboracle.so           the restatement of the reference's algorithms (cg_oracle.cpp,
                         each function cites the reference file:line it follows)
  _ref/libeigen_ref.so   the reference's bundled Eigen CPU path (eigen_ref.cpp)
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
_orc = None
_ref = None


def _p(a) -> Optional[C.c_void_p]:
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def lib():
    global _orc
    if _orc is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            raise ImportError(f"{path} missing: run `make -C oracle`")
        _orc = C.CDLL(str(path))
        vp, i32, i64, f64 = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        sig = {
            "orc_spmv_csr_f32": [i32, vp, vp, vp, i64, i32, vp, i32, i32, vp, i32],
            "orc_spmv_csr_f64": [i32, vp, vp, vp, i64, i32, vp, i32, i32, vp, i32],
            "orc_spmv_csr_f32f64": [i32, vp, vp, vp, i64, i32, vp, i32, i32, vp, i32],
            "orc_spmv_ell_f32": [i32, i32, vp, vp, i32, vp, i32, i32, vp, i32],
            "orc_spmv_ell_f64": [i32, i32, vp, vp, i32, vp, i32, i32, vp, i32],
            "orc_dot_f32": [i64, i32, vp, i32, vp, i32, vp],
            "orc_dot_f64": [i64, i32, vp, i32, vp, i32, vp],
            "orc_inv_diag_f32": [i32, vp, vp, vp, vp],
            "orc_inv_diag_f64": [i32, vp, vp, vp, vp],
            "orc_cg_csr_f32": [i32, vp, vp, vp, i64, i32, vp, i32, vp, vp, f64, i64, C.c_int, C.c_int, vp, vp],
            "orc_cg_csr_f64": [i32, vp, vp, vp, i64, i32, vp, i32, vp, vp, f64, i64, C.c_int, C.c_int, vp, vp],
            "orc_cg_packed_f32": [i64, vp, vp, vp, vp, vp, vp, vp, f64, i64, C.c_int, vp, vp],
            "orc_cg_packed_f64": [i64, vp, vp, vp, vp, vp, vp, vp, f64, i64, C.c_int, vp, vp],
            "orc_refined_packed": [i64, vp, vp, vp, vp, vp, vp, f64, f64, i64, i32, C.c_int, C.c_int, vp, vp, vp],
            "orc_reliable_packed": [i64, vp, vp, vp, vp, vp, vp, f64, f64, i64, i32, C.c_int, C.c_int, vp, vp, vp],
            "orc_reliable_scaled_packed": [i64, vp, vp, vp, vp, vp, vp, f64, f64, i64, i32, C.c_int, C.c_int, vp, vp,
                                           vp],
            "orc_sddmm_csr_f64": [i32, vp, vp, f64, vp, vp, vp],
            "orc_sddmm_csr_f32": [i32, vp, vp, C.c_float, vp, vp, vp],
        }
        for name, args in sig.items():
            fn = getattr(_orc, name)
            fn.restype = C.c_int
            fn.argtypes = args
        _orc.orc_bf16_round.restype = C.c_float
        _orc.orc_bf16_round.argtypes = [C.c_float]
    return _orc


def ref_lib():
    """The reference's bundled Eigen path; None when it was not built."""
    global _ref
    if _ref is None:
        path = HERE / "_ref" / "libeigen_ref.so"
        if not path.exists():
            return None
        _ref = C.CDLL(str(path))
        vp, i32, i64, f64 = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        for name, res, args in [
            ("eref_threads", C.c_int, []),
            ("eref_cg_csr_f32", C.c_int, [i32, vp, vp, vp, vp, vp, f64, i64, C.c_int, vp, vp]),
            ("eref_cg_csr_f64", C.c_int, [i32, vp, vp, vp, vp, vp, f64, i64, C.c_int, vp, vp]),
            ("eref_spmv_csr_f32", f64, [i32, i32, vp, vp, vp, vp, vp, i32, i32]),
            ("eref_llt_solve", C.c_int, [i32, vp, vp, vp, vp, vp, i64]),
            ("eref_dense_solve", C.c_int, [i32, vp, vp, vp]),
            ("eref_packed_create", vp, [i64, vp, vp, vp, vp]),
            ("eref_packed_destroy", None, [vp]),
            ("eref_packed_cg_f64", f64, [vp, i64, i64, vp, vp, f64, i64, C.c_int, i32, vp, vp]),
        ]:
            fn = getattr(_ref, name)
            fn.restype = res
            fn.argtypes = args
    return _ref


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _b2(a, dt):
    a = np.ascontiguousarray(a, dtype=dt)
    return a.reshape(1, -1) if a.ndim == 1 else a


# ---- restatement -------------------------------------------------------------

def spmv_csr(rows, cols, rp, ci, val, x):
    """y[b] = A[b] x[b] (reference CSRMVKernel_StaticBatches, SparseProductEvaluation.h:43-88)."""
    dt = np.float64 if (np.asarray(val).dtype == np.float64 or np.asarray(x).dtype == np.float64) else np.float32
    v = _b2(val, dt)
    xv = _b2(x, dt)
    ob = max(v.shape[0], xv.shape[0])
    y = np.empty((ob, rows), dt)
    f = lib().orc_spmv_csr_f64 if dt == np.float64 else lib().orc_spmv_csr_f32
    f(rows, _p(_i32(rp)), _p(_i32(ci)), _p(v), v.shape[1], v.shape[0], _p(xv), cols, xv.shape[0], _p(y), ob)
    return y


def spmv_csr_f32_in_f64(rows, cols, rp, ci, val32, x64):
    """FP32 values upcast, FP64 vectors (the refinement residual product)."""
    v = _b2(val32, np.float32)
    xv = _b2(x64, np.float64)
    ob = max(v.shape[0], xv.shape[0])
    y = np.empty((ob, rows), np.float64)
    lib().orc_spmv_csr_f32f64(rows, _p(_i32(rp)), _p(_i32(ci)), _p(v), v.shape[1], v.shape[0], _p(xv), cols,
                              xv.shape[0], _p(y), ob)
    return y


def spmv_ell(rows, cols, indices, values, x):
    """indices/values: (rows, width) or values (b, rows, width); skips index < 0
    (reference ELLPACKMVKernel_StaticBatches, SparseProductEvaluation.h:194-226)."""
    idx = np.ascontiguousarray(np.asarray(indices, np.int32).T)  # [slot][row]
    vals = np.asarray(values)
    dt = np.float64 if (vals.dtype == np.float64 or np.asarray(x).dtype == np.float64) else np.float32
    if vals.ndim == 2:
        vals = vals[None]
    vcm = np.ascontiguousarray(vals.transpose(0, 2, 1), dtype=dt)
    xv = _b2(x, dt)
    ob = max(vcm.shape[0], xv.shape[0])
    y = np.empty((ob, rows), dt)
    f = lib().orc_spmv_ell_f64 if dt == np.float64 else lib().orc_spmv_ell_f32
    f(rows, idx.shape[0], _p(idx), _p(vcm), vcm.shape[0], _p(xv), cols, xv.shape[0], _p(y), ob)
    return y


def dot(x, y):
    """Batched dot (reference ReductionOpsPlugin.inl:279-298); pairwise sums in the input type."""
    dt = np.float64 if np.asarray(x).dtype == np.float64 else np.float32
    xv, yv = _b2(x, dt), _b2(y, dt)
    ob = max(xv.shape[0], yv.shape[0])
    out = np.empty(ob, dt)
    f = lib().orc_dot_f64 if dt == np.float64 else lib().orc_dot_f32
    f(xv.shape[1], ob, _p(xv), xv.shape[0], _p(yv), yv.shape[0], _p(out))
    return out


def squared_norm(x):
    return dot(x, x)


def inv_diag(rows, rp, ci, val):
    v = np.ascontiguousarray(val)
    out = np.empty(rows, v.dtype)
    f = lib().orc_inv_diag_f64 if v.dtype == np.float64 else lib().orc_inv_diag_f32
    f(rows, _p(_i32(rp)), _p(_i32(ci)), _p(v), _p(out))
    return out


def cg_csr(n, rp, ci, val, rhs, tol, max_iter=-1, precond=1, lockstep=True, guess=None):
    """The reference's CG (ConjugateGradient.h:123-206) on a shared-pattern batch.
    Returns (x, iterations per batch, error per batch)."""
    dt = np.float64 if np.asarray(rhs).dtype == np.float64 else np.float32
    v = _b2(val, dt)
    b = _b2(rhs, dt)
    B = max(v.shape[0], b.shape[0])
    if b.shape[0] != B:
        b = np.ascontiguousarray(np.broadcast_to(b, (B, n)))
    g = None if guess is None else np.ascontiguousarray(np.broadcast_to(_b2(guess, dt), (B, n)))
    x = np.empty((B, n), dt)
    it = np.empty(B, np.int64)
    err = np.empty(B, np.float64)
    f = lib().orc_cg_csr_f64 if dt == np.float64 else lib().orc_cg_csr_f32
    f(n, _p(_i32(rp)), _p(_i32(ci)), _p(v), v.shape[1], v.shape[0], _p(b), B, _p(g), _p(x), float(tol), int(max_iter),
      int(precond), 1 if lockstep else 0, _p(it), _p(err))
    return x, it, err


def cg_packed(row_off, rp, ci, val, rhs, tol, max_iter=-1, precond=1, guess=None):
    """Per-system reference CG over a packed block-diagonal batch."""
    dt = np.float64 if np.asarray(rhs).dtype == np.float64 else np.float32
    ro = np.ascontiguousarray(row_off, np.int64)
    v = np.ascontiguousarray(val, dt)
    b = np.ascontiguousarray(rhs, dt)
    g = None if guess is None else np.ascontiguousarray(guess, dt)
    x = np.empty_like(b)
    S = ro.size - 1
    it = np.empty(S, np.int64)
    err = np.empty(S, np.float64)
    f = lib().orc_cg_packed_f64 if dt == np.float64 else lib().orc_cg_packed_f32
    f(S, _p(ro), _p(_i32(rp)), _p(_i32(ci)), _p(v), _p(b), _p(g), _p(x), float(tol), int(max_iter), int(precond),
      _p(it), _p(err))
    return x, it, err


def refined_packed(row_off, rp, ci, val32, rhs64, inner_tol, outer_tol, max_inner=-1, max_outer=20, precond=1,
                   bf16_inner=False):
    """FP64 iterative refinement around the FP32 inner PCG, per system.
    Returns (x, outer steps, inner iterations, final relative residual)."""
    ro = np.ascontiguousarray(row_off, np.int64)
    b = np.ascontiguousarray(rhs64, np.float64)
    x = np.empty_like(b)
    S = ro.size - 1
    outer = np.empty(S, np.int32)
    inner = np.empty(S, np.int64)
    err = np.empty(S, np.float64)
    lib().orc_refined_packed(S, _p(ro), _p(_i32(rp)), _p(_i32(ci)), _p(np.ascontiguousarray(val32, np.float32)), _p(b),
                             _p(x), float(inner_tol), float(outer_tol), int(max_inner), int(max_outer), int(precond),
                             1 if bf16_inner else 0, _p(outer), _p(inner), _p(err))
    return x, outer, inner, err


def reliable_packed(row_off, rp, ci, val32, rhs64, tol, delta=0.01, max_iter=-1, max_updates=1000, precond=1,
                    bf16_inner=False, scaled=True):
    """FP32 CG with FP64 reliable updates, per system; scaled=True is the
    Jacobi-scaled form of the CUDA fast path, scaled=False explicit Jacobi PCG.
    Returns (x, FP32 iterations, replacements, final FP64 relative residual)."""
    ro = np.ascontiguousarray(row_off, np.int64)
    b = np.ascontiguousarray(rhs64, np.float64)
    x = np.empty_like(b)
    S = ro.size - 1
    it = np.empty(S, np.int64)
    up = np.empty(S, np.int32)
    err = np.empty(S, np.float64)
    f = lib().orc_reliable_scaled_packed if scaled else lib().orc_reliable_packed
    f(S, _p(ro), _p(_i32(rp)), _p(_i32(ci)), _p(np.ascontiguousarray(val32, np.float32)), _p(b), _p(x), float(tol),
      float(delta), int(max_iter), int(max_updates), int(precond), 1 if bf16_inner else 0, _p(it), _p(up), _p(err))
    return x, it, up, err


def sddmm_csr(rows, rp, ci, u, v, alpha=1.0):
    """alpha * u_i v_j on the pattern (reference sparse outer product)."""
    dt = np.float64 if np.asarray(u).dtype == np.float64 else np.float32
    u = np.ascontiguousarray(u, dt)
    v = np.ascontiguousarray(v, dt)
    out = np.empty(len(ci), dt)
    if dt == np.float64:
        lib().orc_sddmm_csr_f64(rows, _p(_i32(rp)), _p(_i32(ci)), float(alpha), _p(u), _p(v), _p(out))
    else:
        lib().orc_sddmm_csr_f32(rows, _p(_i32(rp)), _p(_i32(ci)), float(alpha), _p(u), _p(v), _p(out))
    return out


def bf16_round(a):
    """Round-to-nearest-even to bfloat16, returned as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) & 0xFFFF0000).astype(np.uint32)
    nonfinite = (a.view(np.uint32) & 0x7F800000) == 0x7F800000
    r = np.where(nonfinite, a.view(np.uint32) & 0xFFFF0000 | np.where(np.isnan(a), 0x00400000, 0), r).astype(np.uint32)
    return r.view(np.float32)


# ---- reference build (bundled Eigen) -------------------------------------------

def eigen_cg(n, rp, ci, val32, rhs, tol, max_iter=-1, precond=1):
    """Eigen ConjugateGradient<SparseMatrix<T, RowMajor>, Lower|Upper, Identity|Diagonal>;
    T from rhs dtype. Returns (x, iterations, error)."""
    R = ref_lib()
    if R is None:
        raise RuntimeError("oracle/_ref/libeigen_ref.so was not built")
    dt = np.float64 if np.asarray(rhs).dtype == np.float64 else np.float32
    b = np.ascontiguousarray(rhs, dt)
    x = np.empty_like(b)
    it = C.c_int64()
    err = C.c_double()
    f = R.eref_cg_csr_f64 if dt == np.float64 else R.eref_cg_csr_f32
    f(n, _p(_i32(rp)), _p(_i32(ci)), _p(np.ascontiguousarray(val32, np.float32)), _p(b), _p(x), float(tol),
      int(max_iter), int(precond), C.byref(it), C.byref(err))
    return x, it.value, err.value


def eigen_llt(n, rp, ci, val32, rhs64, col_base=0):
    """FP64 SimplicialLLT solve (truth for SPD systems)."""
    R = ref_lib()
    if R is None:
        raise RuntimeError("oracle/_ref/libeigen_ref.so was not built")
    b = np.ascontiguousarray(rhs64, np.float64)
    x = np.empty_like(b)
    rc = R.eref_llt_solve(n, _p(_i32(rp)), _p(_i32(ci)), _p(np.ascontiguousarray(val32, np.float32)), _p(b), _p(x),
                          int(col_base))
    if rc != 0:
        raise RuntimeError("SimplicialLLT failed")
    return x


def eigen_dense_solve(A, b):
    R = ref_lib()
    if R is None:
        raise RuntimeError("oracle/_ref/libeigen_ref.so was not built")
    A = np.ascontiguousarray(A, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    x = np.empty_like(b)
    R.eref_dense_solve(A.shape[0], _p(A), _p(b), _p(x))
    return x


def eigen_spmv_seconds(rows, cols, rp, ci, val32, x32, reps, nthreads=0):
    R = ref_lib()
    y = np.empty(rows, np.float32)
    t = R.eref_spmv_csr_f32(rows, cols, _p(_i32(rp)), _p(_i32(ci)), _p(np.ascontiguousarray(val32, np.float32)),
                            _p(np.ascontiguousarray(x32, np.float32)), _p(y), int(reps), int(nthreads))
    return y, t


class EigenPacked:
    """A packed batch of systems as Eigen FP64 row-major matrices (setup untimed)."""

    def __init__(self, row_off, rp, ci, val32):
        R = ref_lib()
        if R is None:
            raise RuntimeError("oracle/_ref/libeigen_ref.so was not built")
        self.R = R
        self.row_off = np.ascontiguousarray(row_off, np.int64)
        self.h = R.eref_packed_create(self.row_off.size - 1, _p(self.row_off), _p(_i32(rp)), _p(_i32(ci)),
                                      _p(np.ascontiguousarray(val32, np.float32)))

    def solve(self, s0, s1, b64, x64, tol, max_iter=-1, precond=1, nthreads=0):
        """Solves systems [s0, s1); returns (seconds, iterations, errors)."""
        it = np.empty(s1 - s0, np.int64)
        err = np.empty(s1 - s0, np.float64)
        t = self.R.eref_packed_cg_f64(self.h, s0, s1, _p(b64), _p(x64), float(tol), int(max_iter), int(precond),
                                      int(nthreads), _p(it), _p(err))
        return t, it, err

    def __del__(self):
        try:
            self.R.eref_packed_destroy(self.h)
        except Exception:
            pass


def ref_threads() -> int:
    R = ref_lib()
    return int(R.eref_threads()) if R is not None else 0
