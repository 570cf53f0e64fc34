"""Device memory through the library's block cache: solvers, matrices and work
buffers built and released per call (the reference's CG benchmark pattern,
benchmarks/conjugate_gradient/Implementation_cuMat.cu) reuse cached blocks
that still hold an earlier owner's data; results must not depend on it."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from cumat_b200 import problems as P  # noqa: E402
from oracle import oracle as O  # noqa: E402


def cm():
    import cumat_b200
    return cumat_b200


def _solve(m, pr, b, dev):
    A = m.SparseMatrix(m.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(pr.val)
    cg = m.ConjugateGradient(A).setTolerance(1e-5)
    x = cg.solve(torch.from_numpy(b).to(dev)).cpu().numpy()
    return x, cg.iterations()


def _poison(m, n, dev):
    # a matrix and solver whose buffers hold NaN, released before the next
    # build so that their blocks go back to the cache dirty
    pr = P.poisson2d(n, 9)
    A = m.SparseMatrix(m.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(
        np.full(pr.nnz, np.nan, np.float32))
    cg = m.ConjugateGradient(A).setTolerance(1e-5).setMaxIterations(3)
    cg.solve(torch.full((pr.n,), float("nan"), device=dev))
    del cg, A


def test_rebuilt_solvers_reuse_dirty_blocks(cuda):
    m = cm()
    cases = [P.poisson2d(g, 3) for g in (60, 100, 200)]
    first = {}
    for rep in range(3):
        for pr in cases:
            _poison(m, 150, cuda)
            x, it = _solve(m, pr, pr.b, cuda)
            if pr.n not in first:
                first[pr.n] = (x, it)
                _, it_o, _ = O.cg_csr(pr.n, pr.row_ptr, pr.col, pr.val, pr.b, 1e-5, -1, 1)
                assert abs(it - int(it_o[0])) <= 2
            else:
                x0, it0 = first[pr.n]
                assert it == it0 and np.array_equal(x, x0), (pr.n, rep)
            assert np.all(np.isfinite(x))
    assert m.Context.current().device_errors() == 0


def test_reductions_and_products_after_dirty_blocks(cuda):
    m = cm()
    rng = np.random.default_rng(5)
    a = rng.uniform(-1, 1, (4, 300, 500))
    x = torch.from_numpy(a).to(cuda)
    ref = m.reduce(x, "sum", ("cols", "batches")).cpu().numpy()
    pr = P.poisson2d(300, 2)
    A = m.SparseMatrix(m.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(pr.val)
    v = torch.from_numpy(pr.b).to(cuda)
    y0 = A.transposed_product(v).cpu().numpy()
    for _ in range(3):
        _poison(m, 200, cuda)
        assert np.array_equal(m.reduce(x, "sum", ("cols", "batches")).cpu().numpy(), ref)
        B = m.SparseMatrix(m.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(pr.val)
        assert np.array_equal(B.transposed_product(v).cpu().numpy(), y0)
        del B
