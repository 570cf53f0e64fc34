"""The C++ facade (include/cuMat/*): the reference's own test cases for this
path, written in C++ against the cuMat-named API (tests/cpp/test_facade.cpp).
CPU: the program compiles and links against libcumat_cg.so with g++ alone
(no CUDA runtime of its own) and fails loudly without a GPU. GPU: every case
passes."""
import os
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
LIBDIR = ROOT / "cumat_b200" / "lib"
SRC = ROOT / "tests" / "cpp" / "test_facade.cpp"
OUT = ROOT / "_build" / "test_facade"


def _compile() -> Path:
    if not (LIBDIR / "libcumat_cg.so").exists():
        pytest.skip("libcumat_cg.so not built")
    cxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else shutil.which("g++")
    OUT.parent.mkdir(exist_ok=True)
    cmd = [cxx, "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"), str(SRC),
           "-L", str(LIBDIR), "-lcumat_cg", f"-Wl,-rpath,{LIBDIR}", "-o", str(OUT)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return OUT


def _run(exe: Path, env=None):
    return subprocess.run([str(exe)], capture_output=True, text=True, timeout=600, env=env)


def test_facade_compiles_without_cuda_runtime():
    exe = _compile()
    out = subprocess.run(["ldd", str(exe)], capture_output=True, text=True).stdout
    assert "libcumat_cg.so" in out and "libcudart" not in out


def test_facade_fails_loudly_without_gpu():
    exe = _compile()
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = _run(exe, env)
    assert r.returncode != 0
    assert "FAIL CSR Matrix-Vector Product" in r.stdout and "CUDA error" in r.stdout


@pytest.mark.gpu
def test_facade_reference_cases(cuda):
    exe = _compile()
    r = _run(exe)
    assert r.returncode == 0, r.stdout + r.stderr
    passed = [line for line in r.stdout.splitlines() if line.startswith("PASS ")]
    assert len(passed) >= 23
    assert "0 failed" in r.stdout
