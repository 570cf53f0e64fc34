"""ctypes binding of the C ABI in include/cumat_cg.h (libcumat_cg.so).

The shared library is built in-tree by ``cumat_b200.build``. There is no
fallback: if it is missing or fails to load, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libcumat_cg.so"

# element types / formats / enums (include/cumat_cg.h)
F32, F64, BF16 = 0, 1, 2
CSR, ELLPACK, CSC, BSR = 0, 1, 2, 3
PRECOND_IDENTITY, PRECOND_JACOBI = 0, 1
ASSIGN, ADD, SUB = 0, 1, 2
SOLVE_CONVERGED, SOLVE_MAX_ITER, SOLVE_ZERO_RHS, SOLVE_BREAKDOWN, SOLVE_NON_FINITE = 0, 1, 2, 3, 4
PATH_AUTO, PATH_PERSISTENT, PATH_GRID, PATH_PERSISTENT_GLOBAL = 0, 1, 2, 3
REFINE_RELIABLE, REFINE_RESTART = 0, 1
REDUCE_SUM, REDUCE_PROD, REDUCE_MIN, REDUCE_MAX = 0, 1, 2, 3
AXIS_ROW, AXIS_COLUMN, AXIS_BATCH = 1, 2, 4
STATUS_NAMES = {0: "OK", 1: "INVALID_ARGUMENT", 2: "CUDA", 3: "OUT_OF_MEMORY", 4: "NOT_SUPPORTED", 5: "INTERNAL"}

_vp = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64
_f64 = C.c_double
_pi32 = C.POINTER(C.c_int32)
_pi64 = C.POINTER(C.c_int64)
_pf64 = C.POINTER(C.c_double)

# name -> (restype, argtypes)
SIGNATURES = {
    "cmcg_last_error_string": (C.c_char_p, []),
    "cmcg_version": (_i32, []),
    "cmcg_launch_count": (_i64, []),
    "cmcg_ctx_create": (_i32, [_i32, _vp, C.POINTER(_vp)]),
    "cmcg_ctx_destroy": (_i32, [_vp]),
    "cmcg_ctx_synchronize": (_i32, [_vp]),
    "cmcg_ctx_stream": (_i32, [_vp, C.POINTER(_vp)]),
    "cmcg_ctx_device_errors": (_i32, [_vp, _pi32]),
    "cmcg_device_alloc": (_i32, [_vp, _i64, C.POINTER(_vp)]),
    "cmcg_device_free": (_i32, [_vp, _vp]),
    "cmcg_memcpy": (_i32, [_vp, _vp, _vp, _i64, _i32]),
    "cmcg_memset_zero": (_i32, [_vp, _vp, _i64]),
    "cmcg_pattern_create_csr": (_i32, [_vp, _i32, _i32, _i64, _vp, _vp, _i32, C.POINTER(_vp)]),
    "cmcg_pattern_create_ell": (_i32, [_vp, _i32, _i32, _i32, _vp, _i32, C.POINTER(_vp)]),
    "cmcg_pattern_create_csc": (_i32, [_vp, _i32, _i32, _i64, _vp, _vp, _i32, C.POINTER(_vp)]),
    "cmcg_pattern_create_bsr": (_i32, [_vp, _i32, _i32, _i32, _i64, _vp, _vp, _i32, C.POINTER(_vp)]),
    "cmcg_pattern_set_systems": (_i32, [_vp, _i64, _vp]),
    "cmcg_pattern_info": (_i32, [_vp, _pi32, _pi32, _pi64, _pi32, _pi64, _pi32]),
    "cmcg_pattern_download": (_i32, [_vp, _vp, _vp]),
    "cmcg_pattern_destroy": (_i32, [_vp]),
    "cmcg_matrix_create": (_i32, [_vp, _i32, _i32, C.POINTER(_vp)]),
    "cmcg_matrix_set_values": (_i32, [_vp, _i32, _vp, _i32]),
    "cmcg_matrix_get_values": (_i32, [_vp, _vp]),
    "cmcg_matrix_info": (_i32, [_vp, _pi32, _pi32]),
    "cmcg_matrix_destroy": (_i32, [_vp]),
    "cmcg_spmv": (_i32, [_vp, _i32, _vp, _i32, _vp, _i32]),
    "cmcg_spmv_transposed": (_i32, [_vp, _i32, _vp, _i32, _vp, _i32]),
    "cmcg_matrix_to_dense": (_i32, [_vp, _vp, _i32]),
    "cmcg_reduce": (_i32, [_vp, _i32, _i32, _i64, _i64, _i64, _i32, _vp, _vp]),
    "cmcg_set_log_callback": (_i32, [_vp, _i32, _vp]),
    "cmcg_matrix_from_dense": (_i32, [_vp, _vp, _i32]),
    "cmcg_dot": (_i32, [_vp, _i32, _i64, _vp, _i32, _vp, _i32, _vp]),
    "cmcg_squared_norm": (_i32, [_vp, _i32, _i64, _vp, _i32, _vp]),
    "cmcg_dot_noalloc": (_i32, [_vp, _i32, _i64, _vp, _i32, _vp, _i32, _vp]),
    "cmcg_lincomb": (_i32, [_vp, _i32, _i64, _i32, _vp, _vp, _vp, _vp, _i32, _i32]),
    "cmcg_sddmm": (_i32, [_vp, _i32, _f64, _vp, _i32, _vp, _i32, _vp, _i32]),
    "cmcg_cg_create": (_i32, [_vp, _i32, C.POINTER(_vp)]),
    "cmcg_cg_destroy": (_i32, [_vp]),
    "cmcg_cg_set_tolerance": (_i32, [_vp, _f64]),
    "cmcg_cg_set_max_iterations": (_i32, [_vp, _i64]),
    "cmcg_cg_get_settings": (_i32, [_vp, _pf64, _pi64]),
    "cmcg_cg_set_path": (_i32, [_vp, _i32]),
    "cmcg_cg_set_refinement": (_i32, [_vp, _i32, _f64]),
    "cmcg_cg_solve": (_i32, [_vp, _i32, _vp, _i32, _vp, _vp]),
    "cmcg_cg_solve_host": (_i32, [_vp, _i32, _vp, _i32, _vp, _vp]),
    "cmcg_cg_iterations": (_i32, [_vp, _pi64]),
    "cmcg_cg_error": (_i32, [_vp, _pf64]),
    "cmcg_cg_system_stats": (_i32, [_vp, _vp, _vp, _vp, _vp]),
    "cmcg_cg_fallbacks": (_i32, [_vp, _vp, _vp]),
    "cmcg_cg_solve_refined": (_i32, [_vp, _vp, _vp, _i32, _vp, _f64, _i32]),
    "cmcg_cg_adjoint": (_i32, [_vp, _vp, _vp, _vp, _i32, _vp, _vp, _f64, _i32]),
}


class CuMatError(RuntimeError):
    """Raised when a C ABI call returns a non-zero status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python cumat_b200/build.py` "
                          "(the library has no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status: int) -> None:
    if status != 0:
        raise CuMatError(status, lib.cmcg_last_error_string().decode(errors="replace"))


def call(name: str, *args) -> None:
    check(getattr(lib, name)(*args))


def launch_count() -> int:
    return int(lib.cmcg_launch_count())
