"""Seeded synthetic problems of the benchmark configurations (host side).

Wraps lib/libcumat_problems.so (csrc/problems.cpp): the reference benchmark's
2D Poisson matrix (benchmarks/conjugate_gradient/Implementation_cuMat.cu:29-41)
and the variable-coefficient finite-volume families built on the same row
ordering. Returns numpy arrays (CSR row_ptr / col / FP32 values).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path
from typing import Optional

import numpy as np

_LIB_PATH = Path(__file__).resolve().parent / "lib" / "libcumat_problems.so"
_lib = None


def _L():
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            from . import build
            build.build_problems()
        _lib = C.CDLL(str(_LIB_PATH))
        vp, i32, i64, f64, u32 = C.c_void_p, C.c_int32, C.c_int64, C.c_double, C.c_uint32
        for name, res, args in [
            ("cmgen_poisson2d_nnz", i64, [i32]),
            ("cmgen_poisson2d", C.c_int, [i32, vp, vp, vp]),
            ("cmgen_uniform_f32", C.c_int, [u32, i64, C.c_float, C.c_float, vp]),
            ("cmgen_fv2d_batch_dims", C.c_int, [i64, i32, i32, u32, vp, vp, vp]),
            ("cmgen_fv2d_batch", C.c_int, [i64, i32, i32, f64, u32, vp, vp, vp, vp, vp, vp]),
            ("cmgen_fv3d_nnz", i64, [i32]),
            ("cmgen_fv3d", C.c_int, [i32, f64, u32, vp, vp, vp, vp]),
            ("cmgen_ell_width", i32, [i32, vp]),
            ("cmgen_csr_to_ell", C.c_int, [i32, vp, vp, vp, i32, vp, vp]),
        ]:
            fn = getattr(_lib, name)
            fn.restype = res
            fn.argtypes = args
    return _lib


def _p(a: np.ndarray) -> C.c_void_p:
    return a.ctypes.data_as(C.c_void_p)


@dataclass
class Problem:
    """A (possibly packed block-diagonal) CSR system with right-hand side(s)."""
    n: int
    row_ptr: np.ndarray      # int32, n + 1
    col: np.ndarray          # int32, nnz
    val: np.ndarray          # float32, nnz
    b: np.ndarray            # float32, n
    row_off: np.ndarray      # int64, n_sys + 1
    xstar: Optional[np.ndarray] = None
    sides: Optional[np.ndarray] = None

    @property
    def nnz(self) -> int:
        return int(self.col.size)

    @property
    def n_sys(self) -> int:
        return int(self.row_off.size - 1)

    def system(self, i: int):
        """(row_ptr, col, val) of system i with local indices."""
        r0, r1 = int(self.row_off[i]), int(self.row_off[i + 1])
        k0, k1 = int(self.row_ptr[r0]), int(self.row_ptr[r1])
        return (self.row_ptr[r0:r1 + 1] - k0).astype(np.int32), (self.col[k0:k1] - r0).astype(np.int32), self.val[k0:k1]


def poisson2d(g: int, seed: int = 0) -> Problem:
    """5-point Poisson on a g x g grid (diag 4, off-diagonals -1), b ~ U[-1,1] from mt19937(seed)."""
    L = _L()
    n = g * g
    nnz = int(L.cmgen_poisson2d_nnz(g))
    rp = np.empty(n + 1, np.int32)
    col = np.empty(nnz, np.int32)
    val = np.empty(nnz, np.float32)
    assert L.cmgen_poisson2d(g, _p(rp), _p(col), _p(val)) == 0
    b = uniform(seed, n)
    return Problem(n, rp, col, val, b, np.array([0, n], np.int64))


def uniform(seed: int, n: int, lo: float = -1.0, hi: float = 1.0) -> np.ndarray:
    out = np.empty(n, np.float32)
    assert _L().cmgen_uniform_f32(seed, n, lo, hi, _p(out)) == 0
    return out


def fv2d_batch(n_sys: int, side_lo: int, side_hi: int, sigma: float, seed: int, with_xstar: bool = False) -> Problem:
    """n_sys independent 2D finite-volume systems (kappa = exp(N(0, sigma^2)) per face),
    sides ~ U{side_lo..side_hi}, packed block-diagonally."""
    L = _L()
    sides = np.empty(n_sys, np.int32)
    rows = C.c_int64()
    nnz = C.c_int64()
    rc = L.cmgen_fv2d_batch_dims(n_sys, side_lo, side_hi, seed, _p(sides), C.byref(rows), C.byref(nnz))
    if rc != 0:
        raise ValueError("fv2d_batch: bad sizes")
    n, nz = rows.value, nnz.value
    rp = np.empty(n + 1, np.int32)
    col = np.empty(nz, np.int32)
    val = np.empty(nz, np.float32)
    ro = np.empty(n_sys + 1, np.int64)
    b = np.empty(n, np.float32)
    xs = np.empty(n, np.float32) if with_xstar else None
    rc = L.cmgen_fv2d_batch(n_sys, side_lo, side_hi, float(sigma), seed, _p(rp), _p(col), _p(val), _p(ro), _p(b),
                            _p(xs) if xs is not None else None)
    assert rc == 0
    return Problem(n, rp, col, val, b, ro, xs, sides)


def fv3d(s: int, sigma: float, seed: int) -> Problem:
    """7-point finite-volume system on an s^3 grid, kappa = exp(N(0, sigma^2))."""
    L = _L()
    n = s ** 3
    nnz = int(L.cmgen_fv3d_nnz(s))
    rp = np.empty(n + 1, np.int32)
    col = np.empty(nnz, np.int32)
    val = np.empty(nnz, np.float32)
    b = np.empty(n, np.float32)
    assert L.cmgen_fv3d(s, float(sigma), seed, _p(rp), _p(col), _p(val), _p(b)) == 0
    return Problem(n, rp, col, val, b, np.array([0, n], np.int64))


def csr_to_ell(rows: int, row_ptr: np.ndarray, col: np.ndarray, val: Optional[np.ndarray] = None, width: int = 0):
    """Column-major ELLPACK (returned as (rows, width) arrays), -1 / 0 padding."""
    L = _L()
    if width <= 0:
        width = int(L.cmgen_ell_width(rows, _p(row_ptr)))
    idx = np.empty(rows * width, np.int32)
    v = np.empty(rows * width, np.float32) if val is not None else None
    rc = L.cmgen_csr_to_ell(rows, _p(row_ptr), _p(col), _p(val) if val is not None else None, width, _p(idx),
                            _p(v) if v is not None else None)
    assert rc == 0
    idx = idx.reshape(width, rows).T
    return (idx, v.reshape(width, rows).T) if v is not None else idx
