"""Storage formats beside CSR and ELLPACK through the C ABI: CSC (the
reference's SparsityPattern<CSC>), block CSR (the reference's blocked CG with
a 3x3 block scalar type), the transposed product, and dense <-> sparse
evaluation on a pattern. Known answers from the reference's tests
(tests/golden/reference_kats.json), everything else against the oracle on the
equivalent CSR matrix."""
import json
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp
import torch

pytestmark = pytest.mark.gpu

from cumat_b200 import problems as P  # noqa: E402
from oracle import oracle as O  # noqa: E402

KAT = json.loads((Path(__file__).resolve().parent / "golden" / "reference_kats.json").read_text())


def cm():
    import cumat_b200
    return cumat_b200


def _rand_csr(rows, cols, density, seed):
    rng = np.random.default_rng(seed)
    A = sp.random(rows, cols, density=density, random_state=rng, format="csr", dtype=np.float64)
    A.data = rng.uniform(-1.0, 1.0, A.nnz)
    A.sort_indices()
    return A


def test_kat_csc_sparse_to_dense(cuda):
    m = cm()
    k = KAT["sparse_to_dense_csc"]
    p = m.SparsityPattern.csc(k["rows"], k["cols"], k["JA"], k["IA"])
    A = m.SparseMatrix(p, batches=2).setData(np.stack([k["values_b0"], k["values_b1"]]).astype(np.float32))
    d = A.toDense().cpu().numpy()
    expect = np.array(k["dense_b0"], np.float32)
    assert np.array_equal(d[0], expect) and np.array_equal(d[1], -expect)
    # values come back in the caller's (column) order
    assert np.array_equal(A.getData(), np.stack([k["values_b0"], k["values_b1"]]).astype(np.float32))
    ja, ia = p.download()
    assert ja.tolist() == k["JA"] and ia.tolist() == k["IA"]


def test_kat_csr_sparse_to_dense_and_back(cuda):
    m = cm()
    k = KAT["sparse_to_dense_csr"]
    p = m.SparsityPattern.csr(k["rows"], k["cols"], k["JA"], k["IA"])
    A = m.SparseMatrix(p, batches=2).setData(np.stack([k["values"], k["values_b1"]]).astype(np.float32))
    d = A.toDense().cpu().numpy()
    assert np.array_equal(d[0], np.array(k["dense_b0"], np.float32))
    # dense -> sparse on the same pattern (column-major dense input too)
    B = m.SparseMatrix(p, batches=2).setFromDense(torch.from_numpy(d).to(cuda))
    assert np.array_equal(B.getData(), A.getData())
    dc = A.toDense(row_major=False).cpu().numpy()
    assert np.array_equal(dc, d)


@pytest.mark.parametrize("dt", [torch.float32, torch.float64])
def test_csc_product_and_solve_vs_oracle(cuda, dt):
    m = cm()
    npdt = np.float32 if dt == torch.float32 else np.float64
    Acsr = _rand_csr(700, 500, 0.02, 3)
    Acsc = Acsr.tocsc()
    Acsc.sort_indices()
    p = m.SparsityPattern.csc(700, 500, Acsc.indptr, Acsc.indices)
    A = m.SparseMatrix(p, dtype=dt).setData(Acsc.data.astype(npdt))
    x = np.random.default_rng(4).uniform(-1, 1, 500).astype(npdt)
    y = (A * torch.from_numpy(x).to(cuda)).cpu().numpy()
    ref = O.spmv_csr(700, 500, Acsr.indptr, Acsr.indices, Acsr.data.astype(npdt), x)[0]
    tol = 1e-6 if dt == torch.float32 else 1e-13
    scale = np.abs(Acsr).astype(np.float64) @ np.abs(x.astype(np.float64))
    assert np.all(np.abs(y - ref) <= tol * np.maximum(scale, 1e-30))
    # a CSC Poisson matrix solved by CG equals the CSR solve
    pr = P.poisson2d(48, 5)
    S = sp.csr_matrix((pr.val, pr.col, pr.row_ptr), shape=(pr.n, pr.n)).tocsc()
    S.sort_indices()
    pc = m.SparsityPattern.csc(pr.n, pr.n, S.indptr, S.indices)
    Ac = m.SparseMatrix(pc).setData(S.data.astype(np.float32))
    Ar = m.SparseMatrix(m.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(pr.val)
    b = torch.from_numpy(pr.b).to(cuda)
    cgc = m.ConjugateGradient(Ac).setTolerance(1e-6)
    cgr = m.ConjugateGradient(Ar).setTolerance(1e-6)
    assert np.array_equal(cgc.solve(b).cpu().numpy(), cgr.solve(b).cpu().numpy())
    assert cgc.iterations() == cgr.iterations()


@pytest.mark.parametrize("dt", [torch.float32, torch.float64])
def test_transposed_product_vs_oracle(cuda, dt):
    m = cm()
    npdt = np.float32 if dt == torch.float32 else np.float64
    Acsr = _rand_csr(900, 400, 0.03, 7)
    p = m.SparsityPattern.csr(900, 400, Acsr.indptr, Acsr.indices)
    vals = np.stack([Acsr.data, 2 * Acsr.data]).astype(npdt)
    A = m.SparseMatrix(p, dtype=dt, batches=2).setData(vals)
    x = np.random.default_rng(8).uniform(-1, 1, (2, 900)).astype(npdt)
    y = A.transposed_product(torch.from_numpy(x).to(cuda)).cpu().numpy()
    At = Acsr.T.tocsr()
    At.sort_indices()
    for b in range(2):
        Atb = sp.csr_matrix(((b + 1) * Acsr.data, Acsr.indices, Acsr.indptr), shape=(900, 400)).T.tocsr()
        Atb.sort_indices()
        ref = O.spmv_csr(400, 900, Atb.indptr, Atb.indices, Atb.data.astype(npdt), x[b])[0]
        tol = 1e-6 if dt == torch.float32 else 1e-13
        scale = np.abs(Atb).astype(np.float64) @ np.abs(x[b].astype(np.float64))
        assert np.all(np.abs(y[b] - ref) <= tol * np.maximum(scale, 1e-30))
    # ADD mode accumulates
    out = torch.ones((2, 400), dtype=dt, device=cuda)
    A.transposed_product(torch.from_numpy(x).to(cuda), out=out, mode=m._native.ADD)
    assert np.allclose(out.cpu().numpy(), y + 1, rtol=1e-6, atol=1e-6)


def test_transposed_product_follows_new_values(cuda):
    # the transposed product reads a copy of the values in the transpose's
    # order; a value upload after the first product must reach the next one
    m = cm()
    Acsr = _rand_csr(300, 500, 0.05, 12)
    p = m.SparsityPattern.csr(300, 500, Acsr.indptr, Acsr.indices)
    A = m.SparseMatrix(p).setData(Acsr.data.astype(np.float32))
    x = torch.from_numpy(np.random.default_rng(13).uniform(-1, 1, 300).astype(np.float32)).to(cuda)
    y1 = A.transposed_product(x).cpu().numpy()
    A.setData((-3.0 * Acsr.data).astype(np.float32))
    y2 = A.transposed_product(x).cpu().numpy()
    assert np.allclose(y2, -3.0 * y1, rtol=1e-5, atol=1e-5)
    Atb = sp.csr_matrix(((-3.0 * Acsr.data).astype(np.float32), Acsr.indices, Acsr.indptr), shape=(300, 500)).T.tocsr()
    Atb.sort_indices()
    ref = O.spmv_csr(500, 300, Atb.indptr, Atb.indices, Atb.data, x.cpu().numpy())[0]
    scale = np.abs(Atb).astype(np.float64) @ np.abs(x.cpu().numpy().astype(np.float64))
    assert np.all(np.abs(y2 - ref) <= 1e-6 * np.maximum(scale, 1e-30))


def _bsr_expand(block_rows, B, brp, bci, blocks):
    """The equivalent scalar CSR (rows of a block row in order, entries block by block)."""
    rp, col, val = [0], [], []
    for I in range(block_rows):
        for i in range(B):
            for k in range(brp[I], brp[I + 1]):
                for j in range(B):
                    col.append(bci[k] * B + j)
                    val.append(blocks[k][i][j])
            rp.append(len(col))
    return np.array(rp, np.int32), np.array(col, np.int32), np.array(val, np.float64)


def test_kat_blocked_cg(cuda):
    # the reference's blocked Poisson problem: 3 x 3 blocks of 3 x 3, tol
    # 1e-5, at most 30 iterations: converged, with work done
    m = cm()
    k = KAT["blocked_cg"]
    B = k["block_size"]
    p = m.SparsityPattern.bsr(k["block_rows"], k["block_rows"], B, k["JA"], k["IA"])
    A = m.SparseMatrix(p).setData(np.array(k["blocks"], np.float32).reshape(-1))
    b = np.array(k["b"], np.float32).reshape(-1)
    cg = m.ConjugateGradient(A).setTolerance(k["tol"]).setMaxIterations(k["max_iterations"])
    x = cg.solve(torch.from_numpy(b).to(cuda)).cpu().numpy()
    assert cg.error() < cg.tolerance()
    assert 0 < cg.iterations() < cg.maxIterations()
    rp, col, val = _bsr_expand(k["block_rows"], B, k["JA"], k["IA"], k["blocks"])
    dense = sp.csr_matrix((val, col, rp), shape=(9, 9)).toarray()
    xt = np.linalg.solve(dense, b.astype(np.float64))
    assert np.linalg.norm(x - xt) / np.linalg.norm(xt) < 1e-4
    _, it_o, _ = O.cg_csr(9, rp, col, val.astype(np.float32), b, k["tol"], k["max_iterations"], 1)
    assert abs(cg.iterations() - int(it_o[0])) <= 2
    # values come back as blocks
    assert np.array_equal(A.getData()[0], np.array(k["blocks"], np.float32))


def _block_poisson(g, B, seed):
    """2D Poisson on a g x g grid of B-vector unknowns coupled inside each
    cell: diagonal blocks 5 I + C (C random symmetric, entries in [-0.1,
    0.1], so its eigenvalues exceed -0.1 B >= -0.4), off-diagonal blocks -I:
    the Laplacian (eigenvalues > 0) plus a block diagonal with eigenvalues
    above 0.6, so SPD."""
    rng = np.random.default_rng(seed)
    n = g * g
    brp, bci, blocks = [0], [], []
    for r in range(n):
        x, y = divmod(r, g)
        nb = []
        for dx, dy in ((-1, 0), (0, -1), (0, 0), (0, 1), (1, 0)):
            if 0 <= x + dx < g and 0 <= y + dy < g:
                nb.append((x + dx) * g + (y + dy))
        for c in sorted(nb):
            if c == r:
                C = rng.uniform(-0.1, 0.1, (B, B))
                blocks.append(5 * np.eye(B) + (C + C.T) / 2)
            else:
                blocks.append(-np.eye(B))
            bci.append(c)
        brp.append(len(bci))
    return np.array(brp, np.int32), np.array(bci, np.int32), np.array(blocks)


@pytest.mark.parametrize("B", [2, 3, 4])
def test_bsr_product_and_cg_vs_oracle(cuda, B):
    m = cm()
    g = 40
    brp, bci, blocks = _block_poisson(g, B, B)
    nb = g * g
    p = m.SparsityPattern.bsr(nb, nb, B, brp, bci)
    A = m.SparseMatrix(p).setData(blocks.astype(np.float32).reshape(-1))
    rp, col, val = _bsr_expand(nb, B, brp, bci, blocks)
    n = nb * B
    x = np.random.default_rng(9).uniform(-1, 1, n).astype(np.float32)
    y = (A * torch.from_numpy(x).to(cuda)).cpu().numpy()
    ref = O.spmv_csr(n, n, rp, col, val.astype(np.float32), x)[0]
    scale = sp.csr_matrix((np.abs(val), col, rp), shape=(n, n)) @ np.abs(x.astype(np.float64))
    assert np.all(np.abs(y - ref) <= 1e-6 * scale)
    b = np.random.default_rng(10).uniform(-1, 1, n).astype(np.float32)
    cg = m.ConjugateGradient(A).setTolerance(1e-6)
    xs = cg.solve(torch.from_numpy(b).to(cuda)).cpu().numpy()
    _, it_o, _ = O.cg_csr(n, rp, col, val.astype(np.float32), b, 1e-6, -1, 1)
    assert cg.system_stats()["status"][0] == 0 and abs(cg.iterations() - int(it_o[0])) <= 2
    # mixed precision with FP64 refinement on the block matrix
    A64 = m.SparseMatrix(p, dtype=torch.float64).setData(blocks.reshape(-1))
    cgm = m.ConjugateGradient(A).setTolerance(1e-4)
    b64 = b.astype(np.float64)
    x64 = cgm.solve_refined(torch.from_numpy(b64).to(cuda), outer=A64, outer_tol=1e-10).cpu().numpy()
    S64 = sp.csr_matrix((val, col, rp), shape=(n, n))
    assert np.linalg.norm(b64 - S64 @ x64) / np.linalg.norm(b64) < 1e-10
