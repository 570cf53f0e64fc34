"""Generates the golden fixtures in this directory. Run from the repository root:

    python tests/golden/make_golden.py

* reference_kats.json - the known-answer tests of the reference's own test suite
  for this path, transcribed as data (each entry cites its source file:line in
  the reference repository).
* eigen_golden.npz    - outputs of the reference's bundled Eigen CPU path
  (oracle/_ref/libeigen_ref.so, built from the reference checkout) on small
  seeded problems: CG iteration counts / errors / solutions and FP64 direct
  solutions. These pin the oracle and the CUDA path on machines where the
  reference checkout is absent.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from cumat_b200 import problems as P  # noqa: E402
from oracle import oracle as O  # noqa: E402


def kats() -> dict:
    csr = {"rows": 4, "cols": 5, "JA": [0, 2, 4, 7, 9], "IA": [0, 1, 1, 2, 0, 3, 4, 2, 4],
           "values": [1, 4, 2, 3, 5, 7, 8, 9, 6]}
    ell = {"rows": 4, "cols": 5, "nnzPerRow": 3,
           "indices": [[0, 1, -1], [1, 2, -1], [0, 3, 4], [2, 4, -1]],
           "values": [[1, 4, 666], [2, 3, 666], [5, 7, 8], [9, 6, 666]]}
    x = [2, 5, 3, -4, 1]
    y = [22, 19, -10, 33]
    tri = {"rows": 5, "cols": 5, "JA": [0, 2, 5, 8, 11, 13], "IA": [0, 1, 0, 1, 2, 1, 2, 3, 2, 3, 4, 3, 4]}
    v1 = np.array([-10, 2, 7, -3, 4], np.float64)
    v2 = np.array([8, 4, 8, -6, 3], np.float64)
    mask = np.zeros((5, 5))
    for r in range(5):
        for k in range(tri["JA"][r], tri["JA"][r + 1]):
            mask[r, tri["IA"][k]] = 1
    outer_dense = (np.outer(v1, v2) * mask).tolist()
    return {
        "spmv_csr": {"source": "tests/TestSparseMultOp.cu:70-102", **csr, "x": x, "y": y},
        "spmv_csr_scaled_matrix": {"source": "tests/TestSparseMultOp.cu:104-153", **csr, "scale": 2, "x": x,
                                   "y": [44, 38, -20, 66]},
        "spmv_csr_batched_matrix": {"source": "tests/TestSparseMultOp.cu:155-192", **csr,
                                    "matrix_scales": [1, 2, 3], "x": x, "y_scales": [1, 2, 3], "y": y},
        "spmv_csr_batched_vector": {"source": "tests/TestSparseMultOp.cu:194-233", **csr,
                                    "vector_scales": [1, 2, 3], "x": x, "y_scales": [1, 2, 3], "y": y},
        "spmv_csr_batched_both": {"source": "tests/TestSparseMultOp.cu:235-276", **csr,
                                  "matrix_scales": [1, 2, -1], "vector_scales": [1, 2, 3], "x": x,
                                  "y_scales": [1, 4, -3], "y": y},
        "spmv_ell": {"source": "tests/TestSparseMultOp.cu:278-317 (padding value 666 never read)", **ell, "x": x,
                     "y": y},
        "spmv_ell_batched_both": {"source": "tests/TestSparseMultOp.cu:471-519", **ell,
                                  "matrix_scales": [1, 2, -1], "vector_scales": [1, 2, 3], "x": x,
                                  "y_scales": [1, 4, -3], "y": y},
        "outer_product_on_pattern": {"source": "tests/TestSparseMultOp.cu:9-67", **tri, "u": v1.tolist(),
                                     "v": v2.tolist(), "dense": outer_dense},
        "sparse_to_dense_csr": {"source": "tests/TestSparseMatrix.cu:10-50", **csr,
                                "values_b1": [-1, -4, -2, -3, -5, -7, -8, -9, -6],
                                "dense_b0": [[1, 4, 0, 0, 0], [0, 2, 3, 0, 0], [5, 0, 0, 7, 8], [0, 0, 9, 0, 6]]},
        "sparse_to_dense_csc": {"source": "tests/TestSparseMatrix.cu:53-101", "rows": 4, "cols": 5,
                                "JA": [0, 2, 4, 6, 7, 9], "IA": [0, 2, 0, 1, 1, 3, 2, 2, 3],
                                "values_b0": [1, 5, 4, 2, 3, 9, 7, 8, 6],
                                "values_b1": [-1, -5, -4, -2, -3, -9, -7, -8, -6],
                                "dense_b0": [[1, 4, 0, 0, 0], [0, 2, 3, 0, 0], [5, 0, 0, 7, 8], [0, 0, 9, 0, 6]]},
        "blocked_cg": {"source": "tests/TestBlockedConjugateGradient.cu:244-275 (3x3 blocks, row-major; the "
                                 "reference's float4 rows carry a zero 4th component, left out here)",
                       "block_rows": 3, "block_size": 3, "JA": [0, 2, 5, 7], "IA": [0, 1, 0, 1, 2, 1, 2],
                       "blocks": [[[2, -1, 0], [-1, 2, -1], [0, -1, 2]], [[0, 0, 0], [0, 0, 0], [-1, 0, 0]],
                                  [[0, 0, -1], [0, 0, 0], [0, 0, 0]], [[2, -1, 0], [-1, 2, -1], [0, -1, 2]],
                                  [[0, 0, 0], [0, 0, 0], [-1, 0, 0]], [[0, 0, -1], [0, 0, 0], [0, 0, 0]],
                                  [[2, -1, 0], [-1, 2, -1], [0, -1, 1]]],
                       "b": [[0.1, 0, 0], [0, 0, 0], [0, 0, -0.1]], "tol": 1e-5, "max_iterations": 30},
        "reduce_axes": {"source": "tests/TestReductionOps2.cu:13-158 (sum), TestReductionOps3.cu:70-125 (min, max "
                                  "over all); data[batch][row][col]; 'row' sums over the row index",
                        "data": [[[5, 2, 4, 1], [8, 5, 6, 2], [-5, 0, 3, -9]],
                                 [[11, 0, 0, 3], [-7, -2, -4, 1], [9, 4, 7, -7]]],
                        "sum": {"none": [[[5, 2, 4, 1], [8, 5, 6, 2], [-5, 0, 3, -9]],
                                         [[11, 0, 0, 3], [-7, -2, -4, 1], [9, 4, 7, -7]]],
                                "column": [[[12], [21], [-11]], [[14], [-12], [13]]],
                                "row": [[[8, 7, 13, -6]], [[13, 2, 3, -3]]],
                                "batch": [[[16, 2, 4, 4], [1, 3, 2, 3], [4, 4, 10, -16]]],
                                "row+column": [[[22]], [[15]]],
                                "column+batch": [[[26], [9], [2]]],
                                "row+batch": [[[21, 9, 16, -9]]],
                                "row+column+batch": [[[37]]]},
                        "min_all": -9, "max_all": 11},
        "reduce_prod": {"source": "tests/TestReductionOps3.cu:42-68",
                        "data": [[[1, 2], [1, 1], [-5, 1]], [[2, 1], [-3, -2], [2, 1]]], "prod_all": -240},
        "dot": {"source": "tests/TestReductionOps4.cu:39-63", "x": [[1, 2, 6], [2, 1, 3]], "y": [[5, -2, 8]],
                "out": [49, 32]},
        "squared_norm": {"source": "tests/TestReductionOps4.cu:65-87", "x": [[5, 2, 4, 1], [11, 0, 0, -3]],
                         "out": [46, 130], "norm": [6.782329983125268139064556326626, 11.401754250991379791360490255668]},
    }


def eigen() -> dict:
    if O.ref_lib() is None:
        raise SystemExit("oracle/_ref/libeigen_ref.so is required (make -C oracle with the reference checkout)")
    out = {}
    # configuration 1: 64 x 64 Poisson, b ~ U[-1,1] seed 0, tol 1e-6, max 1000
    pr = P.poisson2d(64, 0)
    for pc, name in [(0, "identity"), (1, "jacobi")]:
        x, it, err = O.eigen_cg(pr.n, pr.row_ptr, pr.col, pr.val, pr.b, 1e-6, 1000, pc)
        out[f"c1_{name}_x"] = x.astype(np.float32)
        out[f"c1_{name}_iters"] = np.int64(it)
        out[f"c1_{name}_err"] = np.float64(err)
    out["c1_llt_x"] = O.eigen_llt(pr.n, pr.row_ptr, pr.col, pr.val, pr.b.astype(np.float64))
    # small packed batch of variable-coefficient systems (sides 8..24, sigma 0.5, seed 12)
    bt = P.fv2d_batch(16, 8, 24, 0.5, 12)
    its, errs, x64 = [], [], np.empty(bt.n)
    for s in range(bt.n_sys):
        rp, ci, v = bt.system(s)
        r0, r1 = bt.row_off[s], bt.row_off[s + 1]
        _, it, err = O.eigen_cg(r1 - r0, rp, ci, v, bt.b[r0:r1], 1e-6, -1, 1)
        its.append(it)
        errs.append(err)
        x64[r0:r1] = O.eigen_llt(r1 - r0, rp, ci, v, bt.b[r0:r1].astype(np.float64))
    out["batch_iters_jacobi_1e-6"] = np.array(its, np.int64)
    out["batch_err_jacobi_1e-6"] = np.array(errs, np.float64)
    out["batch_llt_x"] = x64
    # small 3D system (s = 12, sigma 1, seed 3): FP64 truth and FP64 Jacobi-CG iterations at 1e-10
    p3 = P.fv3d(12, 1.0, 3)
    out["fv3d12_llt_x"] = O.eigen_llt(p3.n, p3.row_ptr, p3.col, p3.val, p3.b.astype(np.float64))
    _, it, err = O.eigen_cg(p3.n, p3.row_ptr, p3.col, p3.val, p3.b.astype(np.float64), 1e-10, -1, 1)
    out["fv3d12_f64_iters_1e-10"] = np.int64(it)
    out["fv3d12_f64_err_1e-10"] = np.float64(err)
    return out


SAMPLE = 4096   # rows at which a full-size FP64 direct solution is kept


def sample_rows(n: int, seed: int) -> np.ndarray:
    return np.sort(np.random.default_rng(seed).choice(n, size=min(n, SAMPLE), replace=False)).astype(np.int64)


def scale_c2() -> dict:
    """Configuration 2: 1024^2 Poisson, b ~ U[-1,1] seed 1, Jacobi-CG to 1e-6."""
    pr = P.poisson2d(1024, 1)
    out = {}
    x32, it32, err32 = O.eigen_cg(pr.n, pr.row_ptr, pr.col, pr.val, pr.b, 1e-6, 4000, 1)
    _, it64, err64 = O.eigen_cg(pr.n, pr.row_ptr, pr.col, pr.val, pr.b.astype(np.float64), 1e-6, 4000, 1)
    _, ito, erro = O.cg_csr(pr.n, pr.row_ptr, pr.col, pr.val, pr.b, 1e-6, 4000, 1)
    xl = O.eigen_llt(pr.n, pr.row_ptr, pr.col, pr.val, pr.b.astype(np.float64))
    idx = sample_rows(pr.n, 21)
    out.update(c2_eigen_f32_iters=np.int64(it32), c2_eigen_f32_err=np.float64(err32),
               c2_eigen_f64_iters=np.int64(it64), c2_eigen_f64_err=np.float64(err64),
               c2_oracle_f32_iters=np.int64(ito[0]), c2_oracle_f32_err=np.float64(erro[0]),
               c2_idx=idx, c2_llt_x=xl[idx], c2_llt_norm=np.float64(np.linalg.norm(xl)),
               c2_eigen_f32_x=x32[idx].astype(np.float32))
    return out


def scale_c3() -> dict:
    """Configuration 3: the 4096-system batch (sides 16..128, sigma 0.5, seed 2),
    Jacobi-CG per system to 1e-6 in FP32 by the oracle."""
    bt = P.fv2d_batch(4096, 16, 128, 0.5, 2)
    _, it, err = O.cg_packed(bt.row_off, bt.row_ptr, bt.col, bt.val, bt.b, 1e-6, -1, 1)
    return {"c3_oracle_iters": it.astype(np.int16), "c3_oracle_err": err.astype(np.float32)}


def scale_c4() -> dict:
    """The precision configuration's 3D system at 64^3 (sigma 1, seed 3)."""
    p3 = P.fv3d(64, 1.0, 3)
    b64 = p3.b.astype(np.float64)
    _, it, err = O.eigen_cg(p3.n, p3.row_ptr, p3.col, p3.val, b64, 1e-10, -1, 1)
    xl = O.eigen_llt(p3.n, p3.row_ptr, p3.col, p3.val, b64)
    idx = sample_rows(p3.n, 43)
    return {"c4_64_eigen_f64_iters": np.int64(it), "c4_64_eigen_f64_err": np.float64(err), "c4_64_idx": idx,
            "c4_64_llt_x": xl[idx], "c4_64_llt_norm": np.float64(np.linalg.norm(xl))}


def scale(parts) -> None:
    path = HERE / "scale_golden.npz"
    out = dict(np.load(path)) if path.exists() else {}
    for part in parts:
        out = {k: v for k, v in out.items() if not k.startswith(part + "_")}
        out.update({"c2": scale_c2, "c3": scale_c3, "c4": scale_c4}[part]())
    np.savez_compressed(path, **out)
    print("wrote", path, sorted(out))


if __name__ == "__main__":
    if O.ref_lib() is None:
        raise SystemExit("oracle/_ref/libeigen_ref.so is required (make -C oracle REF=<reference checkout>)")
    if len(sys.argv) > 1 and sys.argv[1] == "scale":
        scale(sys.argv[2:] or ["c2", "c3", "c4"])
    else:
        (HERE / "reference_kats.json").write_text(json.dumps(kats(), indent=1))
        np.savez_compressed(HERE / "eigen_golden.npz", **eigen())
        print("wrote", HERE / "reference_kats.json", HERE / "eigen_golden.npz")
