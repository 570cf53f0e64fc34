"""Conjugate gradient through the C ABI on the GPU: the reference's CG tests
(tests/TestConjugateGradient.cu), configuration-1 parity with the reference's
bundled Eigen solver and the oracle, packed uneven batches, mixed precision
with FP64 refinement, failure statuses."""
from pathlib import Path

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from cumat_b200 import problems as P  # noqa: E402
from oracle import oracle as O  # noqa: E402

EIG = np.load(Path(__file__).resolve().parent / "golden" / "eigen_golden.npz")
PATHS = [1, 2]  # persistent, grid


def cm():
    import cumat_b200
    return cumat_b200


def _matrix(pr, dtype=torch.float32, systems=False, fmt="csr"):
    m = cm()
    if fmt == "csr":
        p = m.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)
        vals = pr.val
    else:
        idx, vals = P.csr_to_ell(pr.n, pr.row_ptr, pr.col, pr.val)
        p = m.SparsityPattern.ell(pr.n, pr.n, idx)
    if systems:
        p.set_systems(pr.row_off)
    return m.SparseMatrix(p, dtype=dtype).setData(vals)


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("pc,name", [(0, "identity"), (1, "jacobi")])
def test_config1_matches_eigen_and_oracle(cuda, path, pc, name):
    m = cm()
    pr = P.poisson2d(64, 0)
    A = _matrix(pr)
    cg = m.ConjugateGradient(A, m.IdentityPreconditioner if pc == 0 else m.DiagonalPreconditioner)
    cg.setTolerance(1e-6).setMaxIterations(1000).set_path(path)
    x = cg.solve(torch.from_numpy(pr.b).to(cuda)).cpu().numpy()
    _, it_o, err_o = O.cg_csr(pr.n, pr.row_ptr, pr.col, pr.val, pr.b, 1e-6, 1000, pc)
    assert abs(cg.iterations() - int(EIG[f"c1_{name}_iters"])) <= 2
    assert abs(cg.iterations() - int(it_o[0])) <= 2
    assert cg.error() < 1e-6
    xt = EIG["c1_llt_x"]
    assert np.linalg.norm(x - xt) / np.linalg.norm(xt) < 1e-5
    st = cg.system_stats()
    assert st["status"][0] == 0


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("size", [5, 10, 50, 100])
def test_early_out_rhs(cuda, path, size):
    # reference: Conjugate Gradient - Early Out Rhs (TestConjugateGradient.cu:11-26)
    m = cm()
    rng = np.random.default_rng(size)
    A = rng.uniform(-1, 1, (size, size)).astype(np.float32)
    rp = np.arange(0, size * size + 1, size)
    ci = np.tile(np.arange(size), size)
    S = m.SparseMatrix(m.SparsityPattern.csr(size, size, rp, ci)).setData(A.reshape(-1))
    cg = m.ConjugateGradient(S).set_path(path)
    x = cg.solve(torch.zeros(size, device=cuda))
    assert cg.iterations() == 0 and cg.error() == 0 and float(x.abs().sum()) == 0


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("size", [5, 10, 50, 100])
def test_early_out_x(cuda, path, size):
    # reference: Conjugate Gradient - Early Out X (TestConjugateGradient.cu:28-45)
    m = cm()
    rng = np.random.default_rng(size + 1)
    A = rng.uniform(-1, 1, (size, size))
    xt = rng.uniform(-1, 1, size)
    b = A @ xt
    rp = np.arange(0, size * size + 1, size)
    ci = np.tile(np.arange(size), size)
    S = m.SparseMatrix(m.SparsityPattern.csr(size, size, rp, ci), dtype=torch.float64).setData(A.reshape(-1))
    cg = m.ConjugateGradient(S).set_path(path)
    bt = torch.from_numpy(b).to(cuda)
    # b computed on the device so that the guess is exact to the last bit
    bt = S * torch.from_numpy(xt).to(cuda)
    x = cg.solveWithGuess(bt, torch.from_numpy(xt).to(cuda))
    assert cg.iterations() == 0 and cg.error() < 1e-10
    assert np.array_equal(x.cpu().numpy(), xt)


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("size", [5, 10, 50, 100])
def test_solve_dense(cuda, path, size):
    # reference: Conjugate Gradient - Solve Dense (TestConjugateGradient.cu:47-72), double,
    # default tolerance (epsilon), max 10*size iterations. The reference fills A with
    # U(-1,1) + size*I, which is not symmetric; the reference algorithm (the oracle)
    # does not reach epsilon on such matrices, so the matrix here is symmetrised:
    # (R + R^T)/2 + size*I, diagonally dominant and SPD.
    m = cm()
    rng = np.random.default_rng(100 + size)
    R = rng.uniform(-1, 1, (size, size))
    A = (R + R.T) / 2 + size * np.eye(size)
    xt = rng.uniform(-1, 1, size)
    b = A @ xt
    rp = np.arange(0, size * size + 1, size)
    ci = np.tile(np.arange(size), size)
    S = m.SparseMatrix(m.SparsityPattern.csr(size, size, rp, ci), dtype=torch.float64).setData(A.reshape(-1))
    cg = m.ConjugateGradient(S).setMaxIterations(10 * size).set_path(path)
    x = cg.solve(torch.from_numpy(b).to(cuda)).cpu().numpy()
    assert 0 < cg.iterations() < cg.maxIterations()
    assert 0 < cg.error() <= cg.tolerance()
    assert np.allclose(x, xt, rtol=1e-4)
    _, it_o, _ = O.cg_csr(size, rp, ci, A.reshape(-1), b, cg.tolerance(), 10 * size, 1)
    assert abs(cg.iterations() - int(it_o[0])) <= 2


@pytest.mark.parametrize("path", PATHS)
def test_solve_dense_batched(cuda, path):
    # reference: Conjugate Gradient - Solve Dense Batched (TestConjugateGradient.cu:74-100):
    # one matrix, 3 right-hand sides
    m = cm()
    size, batches = 10, 3
    rng = np.random.default_rng(7)
    R = rng.uniform(-1, 1, (size, size))
    A = (R + R.T) / 2 + size * np.eye(size)
    xt = rng.uniform(-1, 1, (batches, size))
    b = xt @ A.T
    rp = np.arange(0, size * size + 1, size)
    ci = np.tile(np.arange(size), size)
    S = m.SparseMatrix(m.SparsityPattern.csr(size, size, rp, ci), dtype=torch.float64).setData(A.reshape(-1))
    cg = m.ConjugateGradient(S).setMaxIterations(10 * size).set_path(path)
    x = cg.solve(torch.from_numpy(b).to(cuda)).cpu().numpy()
    assert x.shape == (3, size)
    assert 0 < cg.iterations() < cg.maxIterations() and 0 < cg.error() <= cg.tolerance()
    assert np.allclose(x, xt, rtol=1e-4)


@pytest.mark.parametrize("path", PATHS)
def test_batched_matrices_per_batch_jacobi(cuda, path):
    m = cm()
    pr = P.poisson2d(20, 3)
    scales = np.array([1.0, 3.0, 0.25], np.float32)
    p = m.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)
    A = m.SparseMatrix(p, batches=3).setData(np.stack([pr.val * s for s in scales]))
    B = np.stack([pr.b, P.uniform(11, pr.n), P.uniform(12, pr.n)])
    cg = m.ConjugateGradient(A).setTolerance(1e-6).set_path(path)
    x = cg.solve(torch.from_numpy(B).to(cuda)).cpu().numpy()
    xo, it_o, err_o = O.cg_csr(pr.n, pr.row_ptr, pr.col, np.stack([pr.val * s for s in scales]), B, 1e-6, -1, 1,
                               lockstep=False)
    st = cg.system_stats()
    assert np.all(np.abs(st["iterations"] - it_o) <= 2)
    assert np.all(st["error"] < 1e-6) and np.all(st["status"] == 0)
    assert np.allclose(x, xo, rtol=0, atol=1e-5 * np.abs(xo).max())


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("fmt", ["csr", "ell"])
def test_packed_uneven_batch_vs_oracle(cuda, path, fmt):
    m = cm()
    bt = P.fv2d_batch(16, 8, 24, 0.5, 12)   # the batch of eigen_golden.npz
    A = _matrix(bt, systems=True, fmt=fmt)
    cg = m.ConjugateGradient(A).setTolerance(1e-6).set_path(path)
    x = cg.solve(torch.from_numpy(bt.b).to(cuda)).cpu().numpy()
    st = cg.system_stats()
    assert np.all(np.abs(st["iterations"] - EIG["batch_iters_jacobi_1e-6"]) <= 2)
    _, it_o, _ = O.cg_packed(bt.row_off, bt.row_ptr, bt.col, bt.val, bt.b, 1e-6, -1, 1)
    assert np.all(np.abs(st["iterations"] - it_o) <= 2)
    assert np.all(st["status"] == 0) and np.all(st["error"] < 1e-6)
    assert cg.iterations() == st["iterations"].max()
    xt = EIG["batch_llt_x"]
    for s in range(bt.n_sys):
        r0, r1 = bt.row_off[s], bt.row_off[s + 1]
        assert np.linalg.norm(x[r0:r1] - xt[r0:r1]) / np.linalg.norm(xt[r0:r1]) < 1e-4


def test_config3_shaped_batch_vs_oracle(cuda):
    # 256 systems with the side range of configuration 3 (16..128)
    m = cm()
    bt = P.fv2d_batch(256, 16, 128, 0.5, 2)
    A = _matrix(bt, systems=True)
    cg = m.ConjugateGradient(A).setTolerance(1e-6)
    cg.solve(torch.from_numpy(bt.b).to(cuda))  # first solve also lays out the sliced values
    before = m.launch_count()
    x = cg.solve(torch.from_numpy(bt.b).to(cuda))
    assert m.launch_count() - before == 1     # the whole batch is one persistent launch
    st = cg.system_stats()
    _, it_o, _ = O.cg_packed(bt.row_off, bt.row_ptr, bt.col, bt.val, bt.b, 1e-6, -1, 1)
    assert np.all(np.abs(st["iterations"] - it_o) <= 2)
    assert np.all(st["status"] == 0) and np.all(st["error"] < 1e-6)
    # true residual of the FP32 solution, checked in FP64
    r = bt.b - O.spmv_csr_f32_in_f64(bt.n, bt.n, bt.row_ptr, bt.col, bt.val, x.cpu().double().numpy())[0]
    for s in range(0, bt.n_sys, 17):
        r0, r1 = bt.row_off[s], bt.row_off[s + 1]
        # recursive residual < 1e-6; the FP32 iterate's true residual drifts a little above it
        assert np.linalg.norm(r[r0:r1]) / np.linalg.norm(bt.b[r0:r1]) < 2e-5


def test_paths_agree_and_are_deterministic(cuda):
    m = cm()
    bt = P.fv2d_batch(8, 8, 16, 0.5, 4)
    A = _matrix(bt, systems=True)
    b = torch.from_numpy(bt.b).to(cuda)
    xs = []
    for path in PATHS:
        cg = m.ConjugateGradient(A).setTolerance(1e-6).set_path(path)
        x1 = cg.solve(b).cpu().numpy()
        x2 = cg.solve(b).cpu().numpy()
        assert np.array_equal(x1, x2)
        xs.append((x1, cg.system_stats()["iterations"]))
    assert np.all(np.abs(xs[0][1] - xs[1][1]) <= 2)
    assert np.allclose(xs[0][0], xs[1][0], atol=1e-5)


def test_solve_host_buffers(cuda):
    m = cm()
    pr = P.poisson2d(32, 0)
    A = _matrix(pr)
    cg = m.ConjugateGradient(A).setTolerance(1e-6)
    xh = cg.solve_host(pr.b)[0]
    xd = cg.solve(torch.from_numpy(pr.b).to(cuda)).cpu().numpy()
    assert np.array_equal(xh, xd)


@pytest.mark.parametrize("path", PATHS)
def test_failure_statuses(cuda, path):
    m = cm()
    pr = P.poisson2d(8, 0)
    # negative definite matrix: p.Ap < 0 -> BREAKDOWN, no NaN in x
    A = m.SparseMatrix(m.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(-pr.val)
    cg = m.ConjugateGradient(A, m.IdentityPreconditioner).setTolerance(1e-6).set_path(path)
    x = cg.solve(torch.from_numpy(pr.b).to(cuda))
    assert cg.system_stats()["status"][0] == 3
    assert torch.isfinite(x).all()
    # NaN in the right-hand side -> NON_FINITE
    b = pr.b.copy()
    b[3] = np.nan
    A2 = _matrix(pr)
    cg2 = m.ConjugateGradient(A2).set_path(path)
    cg2.solve(torch.from_numpy(b).to(cuda))
    assert cg2.system_stats()["status"][0] == 4
    # iteration limit -> MAX_ITER with iterations == limit
    cg3 = m.ConjugateGradient(A2).setTolerance(1e-12).setMaxIterations(5).set_path(path)
    cg3.solve(torch.from_numpy(pr.b).to(cuda))
    st = cg3.system_stats()
    assert st["status"][0] == 1 and st["iterations"][0] == 5 and cg3.iterations() == 5


@pytest.mark.parametrize("inner", [torch.float32, torch.bfloat16])
def test_refined_to_1e10_vs_fp64_truth(cuda, inner):
    m = cm()
    bt = P.fv2d_batch(16, 8, 24, 0.5, 12)
    p = m.SparsityPattern.csr(bt.n, bt.n, bt.row_ptr, bt.col)
    p.set_systems(bt.row_off)
    Ai = m.SparseMatrix(p, dtype=inner).setData(bt.val)
    Ao = m.SparseMatrix(p, dtype=torch.float32).setData(bt.val)
    cg = m.ConjugateGradient(Ai).setTolerance(1e-4).set_refinement(m._native.REFINE_RESTART)
    b64 = bt.b.astype(np.float64)
    x = cg.solve_refined(torch.from_numpy(b64).to(cuda), outer=Ao, outer_tol=1e-10, max_outer=20).cpu().numpy()
    st = cg.system_stats()
    assert np.all(st["status"] == 0), st
    assert np.all(st["error"] < 1e-10)
    xo, outer_o, inner_o, err_o = O.refined_packed(bt.row_off, bt.row_ptr, bt.col, bt.val, b64, 1e-4, 1e-10,
                                                   bf16_inner=(inner == torch.bfloat16))
    assert np.all(np.abs(st["outer"] - outer_o) <= 1)
    xt = EIG["batch_llt_x"]
    for s in range(bt.n_sys):
        r0, r1 = bt.row_off[s], bt.row_off[s + 1]
        assert np.linalg.norm(x[r0:r1] - xt[r0:r1]) / np.linalg.norm(xt[r0:r1]) < 1e-8
    # true FP64 residual
    r = b64 - O.spmv_csr_f32_in_f64(bt.n, bt.n, bt.row_ptr, bt.col, bt.val, x)[0]
    for s in range(bt.n_sys):
        r0, r1 = bt.row_off[s], bt.row_off[s + 1]
        assert np.linalg.norm(r[r0:r1]) / np.linalg.norm(b64[r0:r1]) < 1e-10


def test_reliable_updates_vs_oracle_and_truth(cuda):
    # mixed precision with FP64 residual replacement on systems of the
    # configuration-3 size range (sides 16..128)
    m = cm()
    bt = P.fv2d_batch(24, 16, 128, 0.5, 2)
    p = m.SparsityPattern.csr(bt.n, bt.n, bt.row_ptr, bt.col)
    p.set_systems(bt.row_off)
    A = m.SparseMatrix(p, dtype=torch.float32).setData(bt.val)
    cg = m.ConjugateGradient(A)
    b64 = bt.b.astype(np.float64)
    cg.solve_refined(torch.from_numpy(b64).to(cuda), outer=A, outer_tol=1e-10, max_outer=200)
    before = m.launch_count()
    x = cg.solve_refined(torch.from_numpy(b64).to(cuda), outer=A, outer_tol=1e-10, max_outer=200).cpu().numpy()
    # one persistent launch per CTA size: 1024 threads for the systems above
    # 8192 rows, 512 threads (two CTAs per SM) down to 4097 rows, 256 threads
    # (four per SM) for the others
    assert m.launch_count() - before == 3
    st = cg.system_stats()
    assert np.all(st["status"] == 0) and np.all(st["error"] < 1e-10)
    xo, it_o, up_o, err_o = O.reliable_packed(bt.row_off, bt.row_ptr, bt.col, bt.val, b64, 1e-10)
    # FP32 rounding (tree vs pairwise sums) moves the points where residuals are
    # replaced, so counts agree to a few per cent, not to the iteration
    assert abs(int(st["iterations"].sum()) - int(it_o.sum())) <= 0.05 * it_o.sum()
    assert np.all(np.abs(st["iterations"] - it_o) <= np.maximum(5, 0.15 * it_o))
    assert np.all(np.abs(st["outer"] - up_o) <= 3)
    _, it64, _ = O.cg_packed(bt.row_off, bt.row_ptr, bt.col, bt.val.astype(np.float64), b64, 1e-10)
    assert st["iterations"].sum() <= 1.15 * it64.sum()   # close to plain FP64 CG's count
    r = b64 - O.spmv_csr_f32_in_f64(bt.n, bt.n, bt.row_ptr, bt.col, bt.val, x)[0]
    for s in range(bt.n_sys):
        r0, r1 = bt.row_off[s], bt.row_off[s + 1]
        assert np.linalg.norm(r[r0:r1]) / np.linalg.norm(b64[r0:r1]) < 1e-10
        if s % 6 == 0 and O.ref_lib() is not None:
            rp, ci, v = bt.system(s)
            xt = O.eigen_llt(r1 - r0, rp, ci, v, b64[r0:r1])
            assert np.linalg.norm(x[r0:r1] - xt) / np.linalg.norm(xt) < 1e-8


@pytest.mark.parametrize("inner", [torch.float32, torch.bfloat16])
def test_diagonal_layout_matches_sliced_layout(cuda, monkeypatch, inner):
    # FV stencils have 5 column offsets per system: the mixed kernel reads the
    # scaled values in the diagonal layout; with CUMAT_CG_DIA=0 it reads the
    # sliced layout. Both add every row's products in the same order.
    m = cm()
    bt = P.fv2d_batch(40, 16, 128, 0.5, 23)
    p = m.SparsityPattern.csr(bt.n, bt.n, bt.row_ptr, bt.col)
    p.set_systems(bt.row_off)
    A = m.SparseMatrix(p, dtype=inner).setData(bt.val)
    A64 = m.SparseMatrix(p, dtype=torch.float64).setData(bt.val.astype(np.float64))
    b64 = torch.from_numpy(bt.b.astype(np.float64)).to(cuda)
    cg = m.ConjugateGradient(A)
    x1 = cg.solve_refined(b64, outer=A64, outer_tol=1e-10, max_outer=200).cpu().numpy()
    s1 = cg.system_stats()
    monkeypatch.setenv("CUMAT_CG_DIA", "0")
    cg0 = m.ConjugateGradient(A)
    x0 = cg0.solve_refined(b64, outer=A64, outer_tol=1e-10, max_outer=200).cpu().numpy()
    s0 = cg0.system_stats()
    assert np.array_equal(s1["status"], s0["status"]) and np.array_equal(s1["iterations"], s0["iterations"])
    assert np.array_equal(s1["outer"], s0["outer"]) and np.array_equal(x1, x0, equal_nan=True)
    if inner == torch.bfloat16:
        # BF16 values (8-bit mantissa) are too coarse for systems whose
        # condition number exceeds ~2^8: the statuses report it, identically
        return
    assert np.all(s1["status"] == 0) and np.all(s1["error"] < 1e-10)
    r = b64.cpu().numpy() - O.spmv_csr_f32_in_f64(bt.n, bt.n, bt.row_ptr, bt.col, bt.val, x1)[0]
    for s in range(bt.n_sys):
        r0, r1 = bt.row_off[s], bt.row_off[s + 1]
        assert np.linalg.norm(r[r0:r1]) / np.linalg.norm(bt.b[r0:r1]) < 1e-10


def _tridiag(n, rng):
    """1D finite-volume diffusion with a reaction term 0.05 (Dirichlet ends):
    offsets -1, 0, 1, condition number ~100."""
    k = np.exp(rng.normal(0.0, 0.5, n + 1))
    rp, col, val = [0], [], []
    for i in range(n):
        if i > 0:
            col.append(i - 1); val.append(-k[i])
        col.append(i); val.append(k[i] + k[i + 1] + 0.05)
        if i < n - 1:
            col.append(i + 1); val.append(-k[i + 1])
        rp.append(len(col))
    return np.array(rp, np.int32), np.array(col, np.int32), np.array(val, np.float32)


def test_diagonal_layout_mixed_offset_sets(cuda, monkeypatch):
    # 2D systems (5 offsets, Jacobi-scaled middle diagonal of ones: its values
    # are not loaded) packed with 1D systems (3 offsets stored in 5 diagonal
    # slots, so the middle slot is not the offset-0 diagonal and every value is
    # loaded): both kinds agree bit for bit with the sliced layout
    m = cm()
    rng = np.random.default_rng(31)
    bt = P.fv2d_batch(6, 16, 80, 0.5, 37)
    rps, cols, vals, offs = [bt.row_ptr], [bt.col], [bt.val], list(bt.row_off)
    n, nnz = bt.n, int(bt.row_ptr[-1])
    for m1 in (700, 1500, 2500):
        rp, c, v = _tridiag(m1, rng)
        rps.append(rp[1:] + nnz); cols.append(c + n); vals.append(v)
        n += m1; nnz += int(rp[-1]); offs.append(n)
    row_ptr, col, val = np.concatenate(rps), np.concatenate(cols), np.concatenate(vals)
    row_off = np.array(offs, np.int64)
    b = rng.uniform(-1.0, 1.0, n)
    p = m.SparsityPattern.csr(n, n, row_ptr, col)
    p.set_systems(row_off)
    A = m.SparseMatrix(p, dtype=torch.float32).setData(val)
    A64 = m.SparseMatrix(p, dtype=torch.float64).setData(val.astype(np.float64))
    b64 = torch.from_numpy(b).to(cuda)
    cg = m.ConjugateGradient(A)
    x1 = cg.solve_refined(b64, outer=A64, outer_tol=1e-10, max_outer=200).cpu().numpy()
    s1 = cg.system_stats()
    monkeypatch.setenv("CUMAT_CG_DIA", "0")
    cg0 = m.ConjugateGradient(A)
    x0 = cg0.solve_refined(b64, outer=A64, outer_tol=1e-10, max_outer=200).cpu().numpy()
    s0 = cg0.system_stats()
    assert np.array_equal(s1["iterations"], s0["iterations"]) and np.array_equal(x1, x0)
    assert np.all(s1["status"] == 0) and np.all(s1["error"] < 1e-10)
    r = b - O.spmv_csr_f32_in_f64(n, n, row_ptr, col, val, x1)[0]
    for s in range(len(offs) - 1):
        r0, r1 = offs[s], offs[s + 1]
        assert np.linalg.norm(r[r0:r1]) / np.linalg.norm(b[r0:r1]) < 1e-10


def test_generic_kernels_match_oracle(cuda, monkeypatch):
    # CUMAT_CG_FAST=0 (read when a solver is created) selects the generic
    # shared-memory kernels: explicit Jacobi PCG inside the reliable updates
    m = cm()
    monkeypatch.setenv("CUMAT_CG_FAST", "0")
    bt = P.fv2d_batch(12, 16, 128, 0.5, 9)
    p = m.SparsityPattern.csr(bt.n, bt.n, bt.row_ptr, bt.col)
    p.set_systems(bt.row_off)
    A = m.SparseMatrix(p, dtype=torch.float32).setData(bt.val)
    cg = m.ConjugateGradient(A)
    b64 = bt.b.astype(np.float64)
    cg.solve_refined(torch.from_numpy(b64).to(cuda), outer=A, outer_tol=1e-10, max_outer=200)
    st = cg.system_stats()
    assert np.all(st["status"] == 0) and np.all(st["error"] < 1e-10)
    _, it_o, up_o, _ = O.reliable_packed(bt.row_off, bt.row_ptr, bt.col, bt.val, b64, 1e-10, scaled=False)
    assert abs(int(st["iterations"].sum()) - int(it_o.sum())) <= 0.05 * it_o.sum()
    cgp = m.ConjugateGradient(A).setTolerance(1e-6)
    cgp.solve(torch.from_numpy(bt.b).to(cuda))
    monkeypatch.setenv("CUMAT_CG_FAST", "1")
    cgf = m.ConjugateGradient(A).setTolerance(1e-6)
    cgf.solve(torch.from_numpy(bt.b).to(cuda))
    assert np.all(np.abs(cgp.system_stats()["iterations"] - cgf.system_stats()["iterations"]) <= 2)


@pytest.mark.parametrize("side_hi", [64, 128])   # FP64 vectors all in shared memory / p only
def test_fp64_fast_kernel_vs_oracle(cuda, side_hi):
    m = cm()
    bt = P.fv2d_batch(20, 16, side_hi, 0.5, 13)
    p = m.SparsityPattern.csr(bt.n, bt.n, bt.row_ptr, bt.col)
    p.set_systems(bt.row_off)
    A = m.SparseMatrix(p, dtype=torch.float64).setData(bt.val.astype(np.float64))
    cg = m.ConjugateGradient(A).setTolerance(1e-10)
    b64 = bt.b.astype(np.float64)
    x = cg.solve(torch.from_numpy(b64).to(cuda)).cpu().numpy()
    st = cg.system_stats()
    _, it_o, _ = O.cg_packed(bt.row_off, bt.row_ptr, bt.col, bt.val.astype(np.float64), b64, 1e-10)
    assert np.all(st["status"] == 0) and np.all(np.abs(st["iterations"] - it_o) <= 2)
    r = b64 - O.spmv_csr_f32_in_f64(bt.n, bt.n, bt.row_ptr, bt.col, bt.val, x)[0]
    for s in range(bt.n_sys):
        r0, r1 = bt.row_off[s], bt.row_off[s + 1]
        assert np.linalg.norm(r[r0:r1]) / np.linalg.norm(b64[r0:r1]) < 2e-10


def test_shared_memory_and_global_kernels_agree(cuda):
    m = cm()
    bt = P.fv2d_batch(40, 16, 128, 0.5, 5)
    A = _matrix(bt, systems=True)
    b = torch.from_numpy(bt.b).to(cuda)
    cg1 = m.ConjugateGradient(A).setTolerance(1e-6).set_path(1)
    x1 = cg1.solve(b).cpu().numpy()
    cg2 = m.ConjugateGradient(A).setTolerance(1e-6).set_path(3)
    x2 = cg2.solve(b).cpu().numpy()
    s1, s2 = cg1.system_stats(), cg2.system_stats()
    assert np.all(s1["status"] == 0) and np.all(s2["status"] == 0)
    assert np.all(np.abs(s1["iterations"] - s2["iterations"]) <= 2)
    assert np.allclose(x1, x2, atol=2e-5 * np.abs(x2).max())


def test_solver_follows_value_and_system_changes(cuda):
    # the reference's solver holds a shallow copy of the matrix, so new values
    # are seen by the next solve; the sliced copy here is regathered
    m = cm()
    bt = P.fv2d_batch(6, 8, 20, 0.5, 8)
    p = m.SparsityPattern.csr(bt.n, bt.n, bt.row_ptr, bt.col)
    A = m.SparseMatrix(p).setData(bt.val)
    cg = m.ConjugateGradient(A, m.IdentityPreconditioner).setTolerance(1e-6)
    b = torch.from_numpy(bt.b).to(cuda)
    cg.solve(b)
    assert cg.system_stats()["status"].shape == (1,)
    p.set_systems(bt.row_off)                 # now 6 independent systems
    x1 = cg.solve(b).cpu().numpy()
    assert cg.system_stats()["status"].shape == (6,)
    A.setData(bt.val * 2.0)                   # scaled matrix: solution halves
    x2 = cg.solve(b).cpu().numpy()
    assert np.allclose(x2, x1 / 2, atol=1e-5)


def test_refined_grid_path_single_system(cuda):
    m = cm()
    p3 = P.fv3d(12, 1.0, 3)
    p = m.SparsityPattern.csr(p3.n, p3.n, p3.row_ptr, p3.col)
    Ai = m.SparseMatrix(p, dtype=torch.float32).setData(p3.val)
    cg = m.ConjugateGradient(Ai).setTolerance(1e-4).set_path(2)
    b64 = p3.b.astype(np.float64)
    x = cg.solve_refined(torch.from_numpy(b64).to(cuda), outer_tol=1e-10).cpu().numpy()
    st = cg.system_stats()
    assert st["status"][0] == 0 and st["error"][0] < 1e-10
    xt = EIG["fv3d12_llt_x"]
    assert np.linalg.norm(x - xt) / np.linalg.norm(xt) < 1e-8


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_cooperative_grid_solve_matches_graph_path(cuda, monkeypatch, dtype):
    # the one-launch cooperative grid solve (one CTA per SM) and the CUDA-graph
    # grid solve (four CTAs per SM) differ only in how the partial sums are
    # grouped
    m = cm()
    monkeypatch.setenv("CUMAT_CG_CLUSTER", "0")   # (the cluster solve would take this size)
    pr = P.poisson2d(160, 3)
    A = _matrix(pr, dtype=dtype)
    b = torch.from_numpy(pr.b.astype(np.float64 if dtype == torch.float64 else np.float32)).to(cuda)
    tol = 1e-10 if dtype == torch.float64 else 1e-6
    cg = m.ConjugateGradient(A).setTolerance(tol).set_path(2)
    cg.solve(b)
    before = m.launch_count()
    x1 = cg.solve(b).cpu().numpy()
    assert m.launch_count() - before == 2      # the cooperative solve + the finaliser
    s1 = cg.system_stats()
    monkeypatch.setenv("CUMAT_CG_COOP", "0")
    cg0 = m.ConjugateGradient(A).setTolerance(tol).set_path(2)
    x0 = cg0.solve(b).cpu().numpy()
    s0 = cg0.system_stats()
    assert s1["status"][0] == 0 and abs(int(s1["iterations"][0]) - int(s0["iterations"][0])) <= 1
    rtol = 1e-9 if dtype == torch.float64 else 1e-4
    assert np.linalg.norm(x1 - x0) / np.linalg.norm(x0) < rtol
    # deterministic: the same launch twice gives the same bits
    assert np.array_equal(cg.solve(b).cpu().numpy(), x1)
    _, it_o, _ = O.cg_csr(pr.n, pr.row_ptr, pr.col, pr.val.astype(np.float64) if dtype == torch.float64 else pr.val,
                          pr.b.astype(np.float64) if dtype == torch.float64 else pr.b, tol, -1, 1)
    assert abs(int(s1["iterations"][0]) - int(it_o[0])) <= 2
    assert m.Context.current().device_errors() == 0


def test_cooperative_grid_solve_batched_instances(cuda, monkeypatch):
    # 3 value batches x 2 systems = 6 instances in one cooperative launch
    m = cm()
    monkeypatch.setenv("CUMAT_CG_CLUSTER", "0")   # (the cluster solve would take these sizes)
    bt = P.fv2d_batch(2, 150, 170, 0.5, 17)
    p = m.SparsityPattern.csr(bt.n, bt.n, bt.row_ptr, bt.col)
    p.set_systems(bt.row_off)
    vals = np.concatenate([bt.val, bt.val * 2.0, bt.val * 0.5]).astype(np.float32)
    A = m.SparseMatrix(p, dtype=torch.float32, batches=3).setData(vals)
    b = torch.from_numpy(np.tile(bt.b, 3)).to(cuda)
    cg = m.ConjugateGradient(A).setTolerance(1e-6).set_path(2)
    x = cg.solve(b).cpu().numpy().reshape(3, -1)
    st = cg.system_stats()
    assert st["status"].shape == (6,) and np.all(st["status"] == 0)
    _, it_o, _ = O.cg_packed(bt.row_off, bt.row_ptr, bt.col, bt.val, bt.b, 1e-6)
    # Jacobi CG is invariant to scaling the matrix: the same counts per batch
    for k in range(3):
        assert np.all(np.abs(st["iterations"][2 * k:2 * k + 2] - it_o) <= 2)
    assert np.allclose(x[1], x[0] / 2, rtol=1e-3, atol=1e-5 * np.abs(x[0]).max())
    assert np.allclose(x[2], x[0] * 2, rtol=1e-3, atol=1e-5 * np.abs(x[0]).max())


def test_grid_reliable_updates_packed_vs_oracle(cuda):
    # the grid path's reliable-update solver on packed systems: same method as
    # the persistent kernel, whole-GPU reductions per system
    m = cm()
    bt = P.fv2d_batch(10, 16, 96, 0.5, 21)
    p = m.SparsityPattern.csr(bt.n, bt.n, bt.row_ptr, bt.col)
    p.set_systems(bt.row_off)
    A = m.SparseMatrix(p, dtype=torch.float32).setData(bt.val)
    A64 = m.SparseMatrix(p, dtype=torch.float64).setData(bt.val.astype(np.float64))
    cg = m.ConjugateGradient(A).set_path(2)
    b64 = bt.b.astype(np.float64)
    x = cg.solve_refined(torch.from_numpy(b64).to(cuda), outer=A64, outer_tol=1e-10, max_outer=200).cpu().numpy()
    st = cg.system_stats()
    assert np.all(st["status"] == 0) and np.all(st["error"] < 1e-10)
    _, it_o, up_o, _ = O.reliable_packed(bt.row_off, bt.row_ptr, bt.col, bt.val, b64, 1e-10)
    assert abs(int(st["iterations"].sum()) - int(it_o.sum())) <= 0.05 * it_o.sum()
    assert np.all(np.abs(st["iterations"] - it_o) <= np.maximum(5, 0.15 * it_o))
    assert np.all(np.abs(st["outer"] - up_o) <= 3)
    r = b64 - O.spmv_csr_f32_in_f64(bt.n, bt.n, bt.row_ptr, bt.col, bt.val, x)[0]
    for s in range(bt.n_sys):
        r0, r1 = bt.row_off[s], bt.row_off[s + 1]
        assert np.linalg.norm(r[r0:r1]) / np.linalg.norm(b64[r0:r1]) < 1e-10
    # the persistent kernel on the same batch agrees to the solution tolerance
    xp = m.ConjugateGradient(A).set_path(1).solve_refined(torch.from_numpy(b64).to(cuda), outer=A64,
                                                          outer_tol=1e-10, max_outer=200).cpu().numpy()
    assert np.linalg.norm(x - xp) / np.linalg.norm(xp) < 1e-8


@pytest.mark.parametrize("inner", [torch.float32, torch.bfloat16])
def test_grid_reliable_updates_3d_vs_eigen(cuda, inner):
    m = cm()
    p3 = P.fv3d(12, 1.0, 3)
    p = m.SparsityPattern.csr(p3.n, p3.n, p3.row_ptr, p3.col)
    Ai = m.SparseMatrix(p, dtype=inner).setData(p3.val)
    Ao = m.SparseMatrix(p, dtype=torch.float64).setData(p3.val.astype(np.float64))
    cg = m.ConjugateGradient(Ai).set_path(2)
    b64 = p3.b.astype(np.float64)
    x = cg.solve_refined(torch.from_numpy(b64).to(cuda), outer=Ao, outer_tol=1e-10, max_outer=100).cpu().numpy()
    st = cg.system_stats()
    assert st["status"][0] == 0 and st["error"][0] < 1e-10
    xt = EIG["fv3d12_llt_x"]
    assert np.linalg.norm(x - xt) / np.linalg.norm(xt) < 1e-8
    # FP32 inner: close to plain FP64 CG's iteration count
    if inner == torch.float32:
        assert cg.iterations() <= 1.15 * int(EIG["fv3d12_f64_iters_1e-10"])


def test_grid_refinement_limits_and_restart(cuda):
    m = cm()
    p3 = P.fv3d(12, 1.0, 3)
    p = m.SparsityPattern.csr(p3.n, p3.n, p3.row_ptr, p3.col)
    Ai = m.SparseMatrix(p, dtype=torch.float32).setData(p3.val)
    Ao = m.SparseMatrix(p, dtype=torch.float64).setData(p3.val.astype(np.float64))
    b64 = torch.from_numpy(p3.b.astype(np.float64)).to(cuda)
    xt = EIG["fv3d12_llt_x"]
    # too few residual replacements: MAX_ITER with the folded solution and
    # its true residual reported
    cg = m.ConjugateGradient(Ai).set_path(2)
    x = cg.solve_refined(b64, outer=Ao, outer_tol=1e-10, max_outer=2).cpu().numpy()
    st = cg.system_stats()
    assert st["status"][0] == 1 and st["outer"][0] == 2
    r = p3.b.astype(np.float64) - O.spmv_csr_f32_in_f64(p3.n, p3.n, p3.row_ptr, p3.col, p3.val, x)[0]
    assert np.isclose(st["error"][0], np.linalg.norm(r) / np.linalg.norm(p3.b.astype(np.float64)), rtol=1e-6)
    # iteration cap: stops with MAX_ITER after exactly that many inner steps
    cg2 = m.ConjugateGradient(Ai).set_path(2).setMaxIterations(7)
    cg2.solve_refined(b64, outer=Ao, outer_tol=1e-10, max_outer=100)
    st2 = cg2.system_stats()
    assert st2["status"][0] == 1 and st2["iterations"][0] == 7 and np.isfinite(st2["error"][0])
    # zero rhs: x = 0
    cg3 = m.ConjugateGradient(Ai).set_path(2)
    x3 = cg3.solve_refined(torch.zeros_like(b64), outer=Ao, outer_tol=1e-10)
    assert cg3.system_stats()["status"][0] == 2 and float(x3.abs().max()) == 0.0
    # restart refinement (host-driven inner solves) still available
    cg4 = m.ConjugateGradient(Ai).setTolerance(1e-4).set_path(2).set_refinement(1)
    x4 = cg4.solve_refined(b64, outer=Ao, outer_tol=1e-10).cpu().numpy()
    assert cg4.system_stats()["status"][0] == 0
    assert np.linalg.norm(x4 - xt) / np.linalg.norm(xt) < 1e-8


def test_plain_fp64_cg_matches_eigen_3d(cuda):
    m = cm()
    p3 = P.fv3d(12, 1.0, 3)
    p = m.SparsityPattern.csr(p3.n, p3.n, p3.row_ptr, p3.col)
    A = m.SparseMatrix(p, dtype=torch.float64).setData(p3.val.astype(np.float64))
    for path in PATHS:
        cg = m.ConjugateGradient(A).setTolerance(1e-10).set_path(path)
        x = cg.solve(torch.from_numpy(p3.b.astype(np.float64)).to(cuda)).cpu().numpy()
        assert abs(cg.iterations() - int(EIG["fv3d12_f64_iters_1e-10"])) <= 2
        xt = EIG["fv3d12_llt_x"]
        assert np.linalg.norm(x - xt) / np.linalg.norm(xt) < 1e-8


def test_fp64_diagonal_tiers_match_sliced_and_oracle(cuda, monkeypatch):
    # plain FP64 PCG on stencil patterns runs on the diagonal layout in three
    # CTA tiers (1024 / 512 / 256 threads by system size); with
    # CUMAT_CG_DIA=0 on the sliced layout with one CTA size. The sums are taken
    # in other orders, so counts agree to +-1 and solutions to FP64 rounding.
    m = cm()
    bt = P.fv2d_batch(60, 16, 128, 0.5, 41)
    assert bt.sides.min() ** 2 <= 4096 < 8192 < bt.sides.max() ** 2   # every tier has systems
    p = m.SparsityPattern.csr(bt.n, bt.n, bt.row_ptr, bt.col)
    p.set_systems(bt.row_off)
    A = m.SparseMatrix(p, dtype=torch.float64).setData(bt.val.astype(np.float64))
    b64 = bt.b.astype(np.float64)
    cg = m.ConjugateGradient(A).setTolerance(1e-10)
    x1 = cg.solve(torch.from_numpy(b64).to(cuda)).cpu().numpy()
    s1 = cg.system_stats()
    monkeypatch.setenv("CUMAT_CG_DIA", "0")
    cg0 = m.ConjugateGradient(A).setTolerance(1e-10)
    x0 = cg0.solve(torch.from_numpy(b64).to(cuda)).cpu().numpy()
    s0 = cg0.system_stats()
    assert np.all(s1["status"] == 0) and np.all(s0["status"] == 0)
    assert np.abs(s1["iterations"] - s0["iterations"]).max() <= 1
    _, it_o, _ = O.cg_packed(bt.row_off, bt.row_ptr, bt.col, bt.val.astype(np.float64), b64, 1e-10)
    assert np.abs(s1["iterations"] - it_o).max() <= 2
    for s in range(bt.n_sys):
        r0, r1 = bt.row_off[s], bt.row_off[s + 1]
        assert np.linalg.norm(x1[r0:r1] - x0[r0:r1]) <= 1e-8 * np.linalg.norm(x0[r0:r1])


def test_fp64_diagonal_tiers_mixed_offset_sets(cuda, monkeypatch):
    # 2D (5 offsets) and 1D (3 offsets in 5 diagonal slots) systems in one
    # batch on the plain FP64 diagonal kernel, against the oracle
    m = cm()
    rng = np.random.default_rng(43)
    bt = P.fv2d_batch(5, 16, 80, 0.5, 47)
    rps, cols, vals, offs = [bt.row_ptr], [bt.col], [bt.val], list(bt.row_off)
    n, nnz = bt.n, int(bt.row_ptr[-1])
    for m1 in (300, 5000, 9000):
        rp, c, v = _tridiag(m1, rng)
        rps.append(rp[1:] + nnz); cols.append(c + n); vals.append(v)
        n += m1; nnz += int(rp[-1]); offs.append(n)
    row_ptr, col, val = np.concatenate(rps), np.concatenate(cols), np.concatenate(vals)
    row_off = np.array(offs, np.int64)
    b = rng.uniform(-1.0, 1.0, n)
    p = m.SparsityPattern.csr(n, n, row_ptr, col)
    p.set_systems(row_off)
    A = m.SparseMatrix(p, dtype=torch.float64).setData(val.astype(np.float64))
    cg = m.ConjugateGradient(A).setTolerance(1e-10)
    x = cg.solve(torch.from_numpy(b).to(cuda)).cpu().numpy()
    st = cg.system_stats()
    _, it_o, _ = O.cg_packed(row_off, row_ptr, col, val.astype(np.float64), b, 1e-10)
    assert np.all(st["status"] == 0) and np.abs(st["iterations"] - it_o).max() <= 2
    r = b - O.spmv_csr_f32_in_f64(n, n, row_ptr, col, val, x)[0]
    for s in range(len(offs) - 1):
        r0, r1 = offs[s], offs[s + 1]
        assert np.linalg.norm(r[r0:r1]) / np.linalg.norm(b[r0:r1]) < 2e-10


@pytest.mark.parametrize("kind", ["fp64", "mixed_f32", "mixed_bf16"])
def test_grid_diagonal_layout_matches_sliced(cuda, monkeypatch, kind):
    # the grid path (one 3D system, graph loop) reads the values in the
    # diagonal layout on stencil patterns; the products add the same terms in
    # the same order as the sliced layout, so both runs agree bit for bit
    m = cm()
    monkeypatch.setenv("CUMAT_CG_COOP", "0")
    monkeypatch.setenv("CUMAT_CG_CLUSTER", "0")
    p3 = P.fv3d(32, 1.0, 5)
    pat = m.SparsityPattern.csr(p3.n, p3.n, p3.row_ptr, p3.col)
    A64 = m.SparseMatrix(pat, dtype=torch.float64).setData(p3.val.astype(np.float64))
    A32 = m.SparseMatrix(pat, dtype=torch.float32).setData(p3.val)
    b64 = torch.from_numpy(p3.b.astype(np.float64)).to(cuda)

    def run():
        if kind == "fp64":
            cg = m.ConjugateGradient(A64).setTolerance(1e-10).set_path(2)
            x = cg.solve(b64)
        else:
            Ai = A32 if kind == "mixed_f32" else m.SparseMatrix(pat, dtype=torch.bfloat16).setData(p3.val)
            cg = m.ConjugateGradient(Ai).setTolerance(1e-4).set_path(2)
            x = cg.solve_refined(b64, outer=A32, outer_tol=1e-10, max_outer=60)
        return x.cpu().numpy(), cg.system_stats()

    x1, s1 = run()
    monkeypatch.setenv("CUMAT_CG_DIA", "0")
    x0, s0 = run()
    assert np.array_equal(s1["iterations"], s0["iterations"]) and np.array_equal(s1["status"], s0["status"])
    assert np.array_equal(x1, x0, equal_nan=True)
    if kind == "mixed_bf16":
        return   # (whether BF16 values converge here depends on the conditioning)
    assert s1["status"][0] == 0
    r = p3.b.astype(np.float64) - O.spmv_csr_f32_in_f64(p3.n, p3.n, p3.row_ptr, p3.col, p3.val, x1)[0]
    assert np.linalg.norm(r) / np.linalg.norm(p3.b.astype(np.float64)) < 1.5e-10


@pytest.mark.parametrize("kind", ["fp64", "mixed_f32"])
@pytest.mark.parametrize("cap", [-1, 21])
def test_host_loop_matches_graph_loop(cuda, monkeypatch, kind, cap):
    # CUMAT_CG_GRAPH=0 launches the grid path's iteration kernels from the host
    # (reading the count of running instances back every 16 iterations)
    # instead of through the graph's WHILE node: the same kernels on the same
    # data, so the same bits, iteration counts and statuses, with or without
    # an iteration cap
    m = cm()
    monkeypatch.setenv("CUMAT_CG_COOP", "0")
    monkeypatch.setenv("CUMAT_CG_CLUSTER", "0")
    p3 = P.fv3d(24, 1.0, 7)
    pat = m.SparsityPattern.csr(p3.n, p3.n, p3.row_ptr, p3.col)
    A64 = m.SparseMatrix(pat, dtype=torch.float64).setData(p3.val.astype(np.float64))
    A32 = m.SparseMatrix(pat, dtype=torch.float32).setData(p3.val)
    b64 = torch.from_numpy(p3.b.astype(np.float64)).to(cuda)

    def run():
        if kind == "fp64":
            cg = m.ConjugateGradient(A64).setTolerance(1e-10).setMaxIterations(cap).set_path(2)
            x = cg.solve(b64)
        else:
            cg = m.ConjugateGradient(A32).setTolerance(1e-4).setMaxIterations(cap).set_path(2)
            x = cg.solve_refined(b64, outer=A32, outer_tol=1e-10, max_outer=60)
        return x.cpu().numpy(), cg.system_stats()

    x1, s1 = run()
    monkeypatch.setenv("CUMAT_CG_GRAPH", "0")
    before = m.launch_count()
    x0, s0 = run()
    host_launches = m.launch_count() - before
    assert np.array_equal(s1["iterations"], s0["iterations"]) and np.array_equal(s1["status"], s0["status"])
    assert np.array_equal(x1, x0, equal_nan=True)
    # one launch per kernel per iteration (the graph counts as one)
    assert host_launches >= 3 * int(s0["iterations"].max())
    if cap < 0:
        assert s1["status"][0] == 0
    elif kind == "fp64":
        assert s1["status"][0] == m._native.SOLVE_MAX_ITER and int(s1["iterations"][0]) == cap


@pytest.mark.parametrize("kind", ["fp64", "mixed_f32"])
def test_grid_p_update_fused_or_separate(cuda, monkeypatch, kind):
    # the grid path's product forms p_k itself where the batch's vectors stay
    # in L2 and reads it from a separate p-update kernel otherwise
    # (CUMAT_CG_FUSE forces either); both evaluate M^-1 r + beta p_{k-1} with
    # the same expression, so iterations, statuses and solutions agree bit for
    # bit, with one kernel launch per iteration less when fused
    m = cm()
    monkeypatch.setenv("CUMAT_CG_COOP", "0")
    monkeypatch.setenv("CUMAT_CG_CLUSTER", "0")
    p3 = P.fv3d(24, 1.0, 9)
    pat = m.SparsityPattern.csr(p3.n, p3.n, p3.row_ptr, p3.col)
    A64 = m.SparseMatrix(pat, dtype=torch.float64).setData(p3.val.astype(np.float64))
    A32 = m.SparseMatrix(pat, dtype=torch.float32).setData(p3.val)
    b64 = torch.from_numpy(p3.b.astype(np.float64)).to(cuda)

    def run(fuse):
        monkeypatch.setenv("CUMAT_CG_FUSE", fuse)
        monkeypatch.setenv("CUMAT_CG_GRAPH", "0")   # (host loop: launches counted per kernel)
        if kind == "fp64":
            cg = m.ConjugateGradient(A64).setTolerance(1e-10).set_path(2)
            before = m.launch_count()
            x = cg.solve(b64)
        else:
            cg = m.ConjugateGradient(A32).setTolerance(1e-4).set_path(2)
            before = m.launch_count()
            x = cg.solve_refined(b64, outer=A32, outer_tol=1e-10, max_outer=60)
        x = x.cpu().numpy()
        return x, cg.system_stats(), m.launch_count() - before

    x1, s1, l1 = run("1")
    x0, s0, l0 = run("0")
    assert np.array_equal(s1["iterations"], s0["iterations"]) and np.array_equal(s1["status"], s0["status"])
    assert s1["status"][0] == 0
    assert np.array_equal(x1, x0)
    assert l0 - l1 >= int(s1["iterations"][0])   # one p-update launch per iteration saved


def test_cooperative_solve_forced_on_large_system(cuda, monkeypatch):
    # systems above 2^15 rows take the graph loop unless CUMAT_CG_COOP=2; the
    # cooperative launch stages each CTA's window of p (its rows plus the
    # columns they reach) in shared memory and must agree with the graph loop
    m = cm()
    pr = P.poisson2d(760, 1)
    assert pr.n > (1 << 15)
    A = _matrix(pr)
    b = torch.from_numpy(pr.b).to(cuda)
    monkeypatch.setenv("CUMAT_CG_COOP", "0")
    cg0 = m.ConjugateGradient(A).setTolerance(1e-6).set_path(2)
    x0 = cg0.solve(b).cpu().numpy()
    monkeypatch.setenv("CUMAT_CG_COOP", "2")
    cg2 = m.ConjugateGradient(A).setTolerance(1e-6).set_path(2)
    cg2.solve(b)
    before = m.launch_count()
    x2 = cg2.solve(b).cpu().numpy()
    assert m.launch_count() - before == 2      # the cooperative solve + the finaliser
    s0, s2 = cg0.system_stats(), cg2.system_stats()
    assert s0["status"][0] == 0 and s2["status"][0] == 0
    assert abs(int(s2["iterations"][0]) - int(s0["iterations"][0])) <= 2
    assert np.linalg.norm(x2 - x0) / np.linalg.norm(x0) < 1e-4
    r = pr.b.astype(np.float64) - O.spmv_csr_f32_in_f64(pr.n, pr.n, pr.row_ptr, pr.col, pr.val, x2)[0]
    # the FP32 recursion drifts from the true residual by about eps_f32 *
    # cond(A) times the size of the updates (1.9e-4 measured at 1024^2)
    assert np.linalg.norm(r) / np.linalg.norm(pr.b.astype(np.float64)) < 1e-3
    assert m.Context.current().device_errors() == 0


def test_bf16_values_fall_back_to_fp32(cuda, monkeypatch):
    # BF16 values round the Jacobi-scaled systems by up to 2^-9; on the larger,
    # worse-conditioned systems of this batch the reliable updates stop
    # contracting. Those systems are solved again with the FP32 values and
    # reported per system; every system then meets the FP64 target.
    m = cm()
    bt = P.fv2d_batch(40, 16, 128, 0.5, 23)
    p = m.SparsityPattern.csr(bt.n, bt.n, bt.row_ptr, bt.col)
    p.set_systems(bt.row_off)
    Ai = m.SparseMatrix(p, dtype=torch.bfloat16).setData(bt.val)
    Ao = m.SparseMatrix(p, dtype=torch.float32).setData(bt.val)
    b64 = bt.b.astype(np.float64)
    cg = m.ConjugateGradient(Ai).setTolerance(1e-4)
    x = cg.solve_refined(torch.from_numpy(b64).to(cuda), outer=Ao, outer_tol=1e-10, max_outer=60).cpu().numpy()
    st = cg.system_stats()
    assert np.all(st["status"] == 0) and np.all(st["error"] < 1e-10)
    r = b64 - O.spmv_csr_f32_in_f64(bt.n, bt.n, bt.row_ptr, bt.col, bt.val, x)[0]
    for s in range(bt.n_sys):
        r0, r1 = bt.row_off[s], bt.row_off[s + 1]
        assert np.linalg.norm(r[r0:r1]) / np.linalg.norm(b64[r0:r1]) < 1e-10
    # the same solve without the fallback: exactly the re-solved systems end
    # unconverged, the others are unchanged
    monkeypatch.setenv("CUMAT_CG_BF16_FALLBACK", "0")
    cg0 = m.ConjugateGradient(Ai).setTolerance(1e-4)
    x0 = cg0.solve_refined(torch.from_numpy(b64).to(cuda), outer=Ao, outer_tol=1e-10, max_outer=60).cpu().numpy()
    s0 = cg0.system_stats()
    assert st["fallback"].sum() > 0
    assert np.array_equal(s0["status"] != 0, st["fallback"] == 1)
    assert s0["fallback"].sum() == 0
    for s in np.nonzero(st["fallback"] == 0)[0]:
        r0, r1 = bt.row_off[s], bt.row_off[s + 1]
        assert np.array_equal(x[r0:r1], x0[r0:r1])
