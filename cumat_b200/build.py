"""Builds the native parts in-tree.

* ``cumat_b200/lib/libcumat_cg.so``       - the sm_100a CUDA kernels + C ABI (nvcc)
* ``cumat_b200/lib/libcumat_problems.so`` - seeded synthetic problem generators (g++)
* ``oracle/`` (test infrastructure)       - via ``make -C oracle``

Objects go to ``_build/`` (git-ignored); the shared libraries are git-ignored
too but stay in the tree so they travel with the repository to a GPU host.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "lib"
OBJ = ROOT / "_build"

NVCC = os.environ.get("CUMAT_NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CUMAT_CXX", "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# (no --split-compile: it builds faster but made the mixed-precision solver
# kernel about 13 % slower on the B200)
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                  "-I" + str(ROOT / "include")]

CU_SOURCES = ["runtime.cu", "spmv.cu", "sell.cu", "sparse_ops.cu", "reduce.cu", "cg.cu", "cg_mixed.cu", "cg_plain.cu",
              "cg_coop.cu", "cg_cluster.cu", "lincomb.cu"]
HEADERS = ["common.cuh", "objects.h", "spmv_dev.cuh", "cg_dev.cuh", "tma.cuh", "cg_smem.cuh", "cg_grid.cuh",
           "grid_sync.cuh", "cg_compact.cuh", "cg_plain.cuh", "cg_cluster.cuh"]


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} ({r.returncode})")


def _local_deps(src: Path) -> list[Path]:
    """The source and every header of this tree it includes, transitively."""
    import re
    seen: dict[Path, None] = {}
    todo = [src]
    while todo:
        f = todo.pop()
        if f in seen or not f.exists():
            continue
        seen[f] = None
        for inc in re.findall(r'^\s*#\s*include\s+"([^"]+)"', f.read_text(), re.M):
            todo.append((f.parent / inc).resolve())
    return list(seen)


def build_cuda(verbose: bool = False, ptxas_info: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    LIB.mkdir(exist_ok=True)
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = CSRC / src
        o = OBJ / (src + ".o")
        objs.append(o)
        if _stale(o, _local_deps(s)) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            jobs.append([NVCC] + NVFLAGS + extra + ["-c", str(s), "-o", str(o)])
    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(_run, jobs))
    so = LIB / "libcumat_cg.so"
    if _stale(so, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", str(so)] + [str(o) for o in objs] + ["-lcudart_static"])
    if verbose:
        print("built", so)
    return so


def build_problems() -> Path:
    LIB.mkdir(exist_ok=True)
    so = LIB / "libcumat_problems.so"
    src = CSRC / "problems.cpp"
    if _stale(so, [src]):
        _run([CXX, "-std=c++17", "-O2", "-fPIC", "-shared", "-march=x86-64-v3", "-o", str(so), str(src)])
    return so


def build_oracle() -> None:
    if shutil.which("make") is None:
        raise RuntimeError("make is required to build the oracle")
    cmd = ["make", "-s", "-C", str(ROOT / "oracle"), f"OCXX={CXX}"]
    # the reference checkout, whose bundled Eigen the timed CPU reference is
    # compiled from; absent on hosts that only run the prebuilt libraries
    ref = Path(os.environ.get("CUMAT_REFERENCE", "/root/reference"))
    if (ref / "third-party" / "Eigen" / "Core").exists():
        cmd.append(f"REF={ref}")
    _run(cmd)


def build_all(verbose: bool = False) -> None:
    build_problems()
    build_oracle()
    build_cuda(verbose=verbose)


if __name__ == "__main__":
    build_all(verbose=True)
    if "--ptxas" in sys.argv:
        build_cuda(ptxas_info=True)
