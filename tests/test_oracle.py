"""Pins the CPU oracle: against the reference's own known-answer tests and
against the reference's bundled Eigen CPU path (golden fixtures made by
tests/golden/make_golden.py). CPU only."""
import json
from pathlib import Path

import numpy as np
import pytest

from cumat_b200 import problems as P
from oracle import oracle as O

GOLD = Path(__file__).resolve().parent / "golden"
KAT = json.loads((GOLD / "reference_kats.json").read_text())
EIG = np.load(GOLD / "eigen_golden.npz")


def _csr(k, dt=np.float32):
    return k["rows"], k["cols"], np.array(k["JA"]), np.array(k["IA"]), np.array(k["values"], dt)


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_kat_spmv_csr(dt):
    k = KAT["spmv_csr"]
    rows, cols, rp, ci, v = _csr(k, dt)
    y = O.spmv_csr(rows, cols, rp, ci, v, np.array(k["x"], dt))
    assert np.array_equal(y[0], np.array(k["y"], dt))
    k2 = KAT["spmv_csr_scaled_matrix"]
    y2 = O.spmv_csr(rows, cols, rp, ci, v * k2["scale"], np.array(k2["x"], dt))
    assert np.array_equal(y2[0], np.array(k2["y"], dt))


@pytest.mark.parametrize("case", ["spmv_csr_batched_matrix", "spmv_csr_batched_vector", "spmv_csr_batched_both"])
def test_kat_spmv_csr_batched(case):
    k = KAT[case]
    rows, cols, rp, ci, v = _csr(k)
    ms = k.get("matrix_scales", [1])
    vs = k.get("vector_scales", [1])
    V = np.stack([v * s for s in ms]).astype(np.float32)
    X = np.stack([np.array(k["x"], np.float32) * s for s in vs])
    y = O.spmv_csr(rows, cols, rp, ci, V, X)
    expect = np.stack([np.array(k["y"], np.float32) * s for s in k["y_scales"]])
    assert np.array_equal(y, expect)


@pytest.mark.parametrize("case", ["spmv_ell", "spmv_ell_batched_both"])
def test_kat_spmv_ell(case):
    k = KAT[case]
    ind = np.array(k["indices"], np.int32)
    val = np.array(k["values"], np.float32)
    ms = k.get("matrix_scales", [1])
    vs = k.get("vector_scales", [1])
    V = np.stack([val * s for s in ms])
    X = np.stack([np.array(k["x"], np.float32) * s for s in vs])
    y = O.spmv_ell(k["rows"], k["cols"], ind, V, X)
    expect = np.stack([np.array(k["y"], np.float32) * s for s in k.get("y_scales", [1])])
    assert np.array_equal(y, expect)


def test_kat_dot_norm():
    k = KAT["dot"]
    for dt in (np.float32, np.float64):
        assert np.array_equal(O.dot(np.array(k["x"], dt), np.array(k["y"], dt)), np.array(k["out"], dt))
        assert np.array_equal(O.dot(np.array(k["y"], dt), np.array(k["x"], dt)), np.array(k["out"], dt))
    k = KAT["squared_norm"]
    sq = O.squared_norm(np.array(k["x"], np.float64))
    assert np.array_equal(sq, np.array(k["out"], np.float64))
    assert np.allclose(np.sqrt(sq), k["norm"], rtol=1e-15)


def test_kat_outer_product_on_pattern():
    k = KAT["outer_product_on_pattern"]
    rp, ci = np.array(k["JA"]), np.array(k["IA"])
    vals = O.sddmm_csr(k["rows"], rp, ci, np.array(k["u"]), np.array(k["v"]))
    dense = np.zeros((5, 5))
    for r in range(5):
        for j in range(rp[r], rp[r + 1]):
            dense[r, ci[j]] = vals[j]
    assert np.array_equal(dense, np.array(k["dense"]))


def test_inverse_diagonal_check():
    # zero and missing diagonals give 1 (cwiseInverseCheck)
    rp = np.array([0, 2, 3, 4])
    ci = np.array([0, 1, 0, 2])
    v = np.array([4.0, 1.0, 7.0, 0.0])
    assert np.array_equal(O.inv_diag(3, rp, ci, v), [0.25, 1.0, 1.0])


@pytest.mark.parametrize("pc,name", [(0, "identity"), (1, "jacobi")])
def test_oracle_cg_matches_eigen_config1(pc, name):
    pr = P.poisson2d(64, 0)
    x, it, err = O.cg_csr(pr.n, pr.row_ptr, pr.col, pr.val, pr.b, 1e-6, 1000, pc)
    assert abs(int(it[0]) - int(EIG[f"c1_{name}_iters"])) <= 2
    assert err[0] < 1e-6
    assert abs(err[0] - float(EIG[f"c1_{name}_err"])) < 1e-7
    xt = EIG["c1_llt_x"]
    assert np.linalg.norm(x[0] - xt) / np.linalg.norm(xt) < 1e-5
    assert np.allclose(x[0], EIG[f"c1_{name}_x"], rtol=0, atol=1e-4)


def test_oracle_cg_packed_matches_eigen():
    bt = P.fv2d_batch(16, 8, 24, 0.5, 12)
    x, it, err = O.cg_packed(bt.row_off, bt.row_ptr, bt.col, bt.val, bt.b, 1e-6, -1, 1)
    assert np.all(np.abs(it - EIG["batch_iters_jacobi_1e-6"]) <= 2)
    assert np.all(err < 1e-6)
    xt = EIG["batch_llt_x"]
    for s in range(bt.n_sys):
        r0, r1 = bt.row_off[s], bt.row_off[s + 1]
        assert np.linalg.norm(x[r0:r1] - xt[r0:r1]) / np.linalg.norm(xt[r0:r1]) < 1e-4


def test_oracle_cg_f64_3d_matches_eigen():
    p3 = P.fv3d(12, 1.0, 3)
    x, it, err = O.cg_csr(p3.n, p3.row_ptr, p3.col, p3.val.astype(np.float64), p3.b.astype(np.float64), 1e-10, -1, 1)
    assert abs(int(it[0]) - int(EIG["fv3d12_f64_iters_1e-10"])) <= 2
    xt = EIG["fv3d12_llt_x"]
    assert np.linalg.norm(x[0] - xt) / np.linalg.norm(xt) < 1e-8


def test_oracle_early_outs():
    pr = P.poisson2d(8, 0)
    # zero right-hand side: x = 0, iterations 0, error 0 (ConjugateGradient.h:152-159)
    x, it, err = O.cg_csr(pr.n, pr.row_ptr, pr.col, pr.val, np.zeros(pr.n, np.float32), 1e-6)
    assert it[0] == 0 and err[0] == 0 and not x.any()
    # exact guess: iterations 0 (ConjugateGradient.h:162-171)
    xt = np.random.default_rng(0).uniform(-1, 1, pr.n)
    b = O.spmv_csr(pr.n, pr.n, pr.row_ptr, pr.col, pr.val.astype(np.float64), xt)[0]
    x, it, err = O.cg_csr(pr.n, pr.row_ptr, pr.col, pr.val.astype(np.float64), b, 1e-6, guess=xt)
    assert it[0] == 0 and err[0] < 1e-10 and np.array_equal(x[0], xt)


def test_oracle_lockstep_vs_per_system():
    # lock-stepped batches report one count = the largest per-batch count
    pr = P.poisson2d(16, 0)
    B = np.stack([pr.b, P.uniform(5, pr.n), P.uniform(6, pr.n)])
    V = np.stack([pr.val, pr.val * 2, pr.val * 0.5])
    _, it_l, _ = O.cg_csr(pr.n, pr.row_ptr, pr.col, V, B, 1e-6, -1, 1, lockstep=True)
    _, it_s, err_s = O.cg_csr(pr.n, pr.row_ptr, pr.col, V, B, 1e-6, -1, 1, lockstep=False)
    assert np.all(it_l == it_l[0]) and abs(int(it_l[0]) - int(it_s.max())) <= 1
    assert np.all(err_s < 1e-6)


def test_oracle_refined_reaches_1e10():
    bt = P.fv2d_batch(8, 8, 20, 0.5, 21)
    b64 = bt.b.astype(np.float64)
    for bf16 in (False, True):
        x, outer, inner, err = O.refined_packed(bt.row_off, bt.row_ptr, bt.col, bt.val, b64, 1e-4, 1e-10,
                                                bf16_inner=bf16)
        assert np.all(err < 1e-10), (bf16, err)
        assert np.all(outer >= 2) and np.all(outer <= 8)
        for s in range(bt.n_sys):
            r0, r1 = bt.row_off[s], bt.row_off[s + 1]
            rp, ci, v = bt.system(s)
            xt = O.eigen_llt(r1 - r0, rp, ci, v, b64[r0:r1]) if O.ref_lib() else None
            if xt is not None:
                assert np.linalg.norm(x[r0:r1] - xt) / np.linalg.norm(xt) < 1e-8


def test_bf16_round_matches_torch():
    torch = pytest.importorskip("torch")
    a = np.random.default_rng(3).standard_normal(10000).astype(np.float32) * 100
    a[:4] = [np.inf, -np.inf, 0.0, -0.0]
    ref = torch.from_numpy(a).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(O.bf16_round(a), ref)
    assert O.lib().orc_bf16_round(1.00390625) == ref.dtype.type(torch.tensor(1.00390625).to(torch.bfloat16).float().item())
