"""The C-ABI library loads and exports every symbol include/cumat_cg.h declares;
argument validation that needs no device. CPU only (no compute calls)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "cumat_cg.h"
LIB = ROOT / "cumat_b200" / "lib" / "libcumat_cg.so"


def declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(cmcg_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def native():
    if not LIB.exists():
        pytest.skip("libcumat_cg.so not built (run __graft_entry__.build())")
    from cumat_b200 import _native
    return _native


def test_header_declares_api():
    names = declared()
    for must in ["cmcg_spmv", "cmcg_dot", "cmcg_squared_norm", "cmcg_cg_create", "cmcg_cg_solve",
                 "cmcg_cg_solve_refined", "cmcg_cg_adjoint", "cmcg_pattern_create_csr", "cmcg_pattern_create_ell",
                 "cmcg_sddmm"]:
        assert must in names


def test_library_exports_every_declared_symbol(native):
    lib = C.CDLL(str(LIB))
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB)], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (cmcg_[a-z0-9_]+)", out))
    assert set(declared()) <= exported


def test_ctypes_binding_covers_header(native):
    assert set(native.SIGNATURES) == set(declared())


def test_version_and_error_string(native):
    assert native.lib.cmcg_version() >= 10000
    assert isinstance(native.lib.cmcg_last_error_string(), bytes)


def test_validation_without_device(native):
    L = native.lib
    assert L.cmcg_ctx_create(0, None, None) == 1
    assert b"NULL" in L.cmcg_last_error_string()
    assert L.cmcg_cg_set_tolerance(None, 1e-6) == 1
    assert L.cmcg_spmv(None, 0, None, 1, None, 0) == 1
    assert L.cmcg_pattern_create_csr(None, 4, 4, 0, None, None, 0, None) == 1
    assert L.cmcg_cg_create(None, 1, None) == 1
    assert L.cmcg_lincomb(None, 0, 8, 1, None, None, None, None, 1, 0) == 1
    assert L.cmcg_device_alloc(None, 16, None) == 1
    with pytest.raises(native.CuMatError):
        native.check(L.cmcg_matrix_create(None, 0, 1, None))


def test_product_path_has_no_oracle_dependency():
    # the package never imports, links or loads the oracle
    # no product source names the oracle outside the build script, which only
    # compiles it (comments included: the product does not describe itself in
    # terms of its checker)
    for p in (ROOT / "cumat_b200").rglob("*"):
        if p.suffix in {".py", ".cu", ".cuh", ".h", ".cpp"} and p.name != "build.py":
            assert "oracle" not in p.read_text().lower(), p
    src = "\n".join(p.read_text() for p in (ROOT / "cumat_b200").rglob("*.py") if p.name != "build.py")
    assert "import oracle" not in src and "from oracle" not in src
    out = subprocess.run(["ldd", str(LIB)], capture_output=True, text=True).stdout if LIB.exists() else ""
    assert "oracle" not in out and "eigen_ref" not in out
