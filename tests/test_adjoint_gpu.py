"""Adjoint gradients of x = A^{-1} b (differentiation configuration, scaled
down): dL/db and dL/dA on the pattern for L = 1/2 |x - x*|^2, checked against
FP64 central finite differences (h = 1e-6) and a dense FP64 reference
gradient (numpy / the reference's bundled Eigen)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from cumat_b200 import problems as P  # noqa: E402
from oracle import oracle as O  # noqa: E402


def _dense(bt, s):
    rp, ci, v = bt.system(s)
    n = rp.size - 1
    A = np.zeros((n, n))
    for r in range(n):
        A[r, ci[rp[r]:rp[r + 1]]] = v[rp[r]:rp[r + 1]]
    return A, rp, ci


def test_adjoint_vs_dense_and_finite_differences(cuda):
    from cumat_b200.autograd import SparseSolveOp
    bt = P.fv2d_batch(8, 12, 20, 0.5, 4, with_xstar=True)
    op = SparseSolveOp(bt.n, bt.row_ptr, bt.col, bt.row_off)
    vals = torch.from_numpy(bt.val.astype(np.float64)).to(cuda)
    op.set_values(vals)
    b = torch.from_numpy(bt.b.astype(np.float64)).to(cuda)
    xs = bt.xstar.astype(np.float64)
    x = op.solve(b)
    gx = x - torch.from_numpy(xs).to(cuda)
    gb, gA = op.adjoint(x, gx)
    x, gb, gA = x.cpu().numpy(), gb.cpu().numpy(), gA.cpu().numpy()[0]
    rng = np.random.default_rng(0)
    checked = 0
    for s in range(bt.n_sys):
        r0, r1 = bt.row_off[s], bt.row_off[s + 1]
        A, rp, ci = _dense(bt, s)
        bs = bt.b[r0:r1].astype(np.float64)
        xt = np.linalg.solve(A, bs)
        assert np.linalg.norm(x[r0:r1] - xt) / np.linalg.norm(xt) < 1e-11
        lam = np.linalg.solve(A.T, xt - xs[r0:r1])
        assert np.linalg.norm(gb[r0:r1] - lam) / np.linalg.norm(lam) < 1e-9
        k0 = bt.row_ptr[r0]
        for r in range(r1 - r0):
            for k in range(rp[r], rp[r + 1]):
                assert abs(gA[k0 + k] - (-lam[r] * xt[ci[k]])) <= 1e-9 * np.abs(lam).max() * np.abs(xt).max()
        # central finite differences of L in FP64 (h = 1e-6) on 8 random b and A
        # entries, measured relative to the gradient's scale in this system
        L = lambda xx: 0.5 * np.sum((xx - xs[r0:r1]) ** 2)  # noqa: E731
        h = 1e-6
        gscale = max(np.abs(lam).max(), np.abs(gA[k0:bt.row_ptr[r1]]).max())
        for i in rng.choice(r1 - r0, 4, replace=False):
            e = np.zeros(r1 - r0)
            e[i] = h
            fd = (L(np.linalg.solve(A, bs + e)) - L(np.linalg.solve(A, bs - e))) / (2 * h)
            assert abs(fd - gb[r0 + i]) <= 1e-6 * gscale
            checked += 1
        for kk in rng.choice(rp[-1], 4, replace=False):
            r = int(np.searchsorted(rp, kk, side="right") - 1)
            c = ci[kk]
            Ap, Am = A.copy(), A.copy()
            Ap[r, c] += h
            Am[r, c] -= h
            fd = (L(np.linalg.solve(Ap, bs)) - L(np.linalg.solve(Am, bs))) / (2 * h)
            assert abs(fd - gA[k0 + kk]) <= 1e-6 * gscale
            checked += 1
    assert checked == 64


def test_adjoint_dense_eigen_gradient_32x32(cuda):
    # one 32 x 32 system: the whole dL/dA on the pattern against a dense FP64
    # gradient from the reference's bundled Eigen (PartialPivLU)
    if O.ref_lib() is None:
        pytest.skip("bundled Eigen build not present")
    from cumat_b200.autograd import SparseSolveOp
    bt = P.fv2d_batch(1, 32, 32, 0.5, 4, with_xstar=True)
    op = SparseSolveOp(bt.n, bt.row_ptr, bt.col)
    op.set_values(torch.from_numpy(bt.val.astype(np.float64)).to(cuda))
    b = torch.from_numpy(bt.b.astype(np.float64)).to(cuda)
    x = op.solve(b)
    gb, gA = op.adjoint(x, x - torch.from_numpy(bt.xstar.astype(np.float64)).to(cuda))
    A, rp, ci = _dense(bt, 0)
    xt = O.eigen_dense_solve(A, bt.b.astype(np.float64))
    lam = O.eigen_dense_solve(np.ascontiguousarray(A.T), xt - bt.xstar)
    G = -np.outer(lam, xt)
    ref = np.array([G[r, ci[k]] for r in range(bt.n) for k in range(rp[r], rp[r + 1])])
    got = gA.cpu().numpy()[0]
    assert np.max(np.abs(got - ref)) <= 1e-9 * np.abs(ref).max()
    assert np.allclose(gb.cpu().numpy(), lam, rtol=1e-9, atol=1e-12)


def test_autograd_function_matches_adjoint(cuda):
    from cumat_b200.autograd import SparseSolveOp, sparse_solve
    bt = P.fv2d_batch(3, 6, 8, 0.5, 4, with_xstar=True)
    op = SparseSolveOp(bt.n, bt.row_ptr, bt.col, bt.row_off)
    vals = torch.from_numpy(bt.val.astype(np.float64)).to(cuda).requires_grad_(True)
    b = torch.from_numpy(bt.b.astype(np.float64)).to(cuda).requires_grad_(True)
    xs = torch.from_numpy(bt.xstar.astype(np.float64)).to(cuda)
    x = sparse_solve(vals, b, op)
    loss = 0.5 * ((x - xs) ** 2).sum()
    loss.backward()
    # torch's own finite-difference check of the adjoint (FP64)
    assert torch.autograd.gradcheck(lambda v, bb: sparse_solve(v, bb, op), (vals.detach().requires_grad_(True),
                                                                           b.detach().requires_grad_(True)),
                                    eps=1e-6, atol=1e-6, rtol=1e-5)
    assert vals.grad is not None and b.grad is not None and torch.isfinite(vals.grad).all()


def test_adjoint_config5_shape_vs_sparse_fd(cuda):
    # the differentiation configuration's system size (128 x 128 grids), a
    # small batch; 64 entries checked against FP64 central differences of
    # sparse direct solves (scipy SuperLU)
    sp = pytest.importorskip("scipy.sparse")
    spl = pytest.importorskip("scipy.sparse.linalg")
    from cumat_b200.autograd import SparseSolveOp
    bt = P.fv2d_batch(4, 128, 128, 0.5, 4, with_xstar=True)
    op = SparseSolveOp(bt.n, bt.row_ptr, bt.col, bt.row_off)
    op.set_values(torch.from_numpy(bt.val.astype(np.float64)).to(cuda))
    b = torch.from_numpy(bt.b.astype(np.float64)).to(cuda)
    xs = bt.xstar.astype(np.float64)
    x = op.solve(b)
    gb, gA = op.adjoint(x, x - torch.from_numpy(xs).to(cuda))
    gb, gA = gb.cpu().numpy(), gA.cpu().numpy()[0]
    rng = np.random.default_rng(1)
    h = 1e-6
    for s in range(bt.n_sys):
        r0, r1 = bt.row_off[s], bt.row_off[s + 1]
        rp, ci, v = bt.system(s)
        n = r1 - r0
        A = sp.csr_matrix((v.astype(np.float64), ci, rp), shape=(n, n)).tocsc()
        lu = spl.splu(A)
        bs = bt.b[r0:r1].astype(np.float64)
        L = lambda xx: 0.5 * np.sum((xx - xs[r0:r1]) ** 2)  # noqa: E731
        # |L| ~ 1e5 and kappa ~ 1e4 here, so FP64 central differences carry
        # noise of ~1e-5 absolute; the agreement is measured relative to the
        # gradient's scale (its largest entry in this system)
        k0, k1 = bt.row_ptr[r0], bt.row_ptr[r1]
        gscale = max(np.abs(gb[r0:r1]).max(), np.abs(gA[k0:k1]).max())
        for i in rng.choice(n, 8, replace=False):
            e = np.zeros(n)
            e[i] = h
            fd = (L(lu.solve(bs + e)) - L(lu.solve(bs - e))) / (2 * h)
            assert abs(fd - gb[r0 + i]) <= 1e-6 * gscale
        for kk in rng.choice(rp[-1], 8, replace=False):
            r = int(np.searchsorted(rp, kk, side="right") - 1)
            E = sp.csr_matrix(([h], ([r], [ci[kk]])), shape=(n, n)).tocsc()
            fd = (L(spl.spsolve(A + E, bs)) - L(spl.spsolve(A - E, bs))) / (2 * h)
            assert abs(fd - gA[k0 + kk]) <= 1e-6 * gscale


def test_autograd_broadcast_and_interleaved_forwards(cuda):
    # batched values with a one-batch b: the gradient of b sums over the
    # batches and has b's shape; two forwards on the same op before the first
    # backward: each backward uses its own forward's values
    from cumat_b200.autograd import SparseSolveOp, sparse_solve
    bt = P.fv2d_batch(2, 6, 8, 0.5, 9, with_xstar=True)
    op = SparseSolveOp(bt.n, bt.row_ptr, bt.col, bt.row_off)
    v0 = bt.val.astype(np.float64)
    vals = torch.from_numpy(np.stack([v0, 1.5 * v0])).to(cuda).requires_grad_(True)
    b = torch.from_numpy(bt.b.astype(np.float64)).to(cuda).requires_grad_(True)
    x = sparse_solve(vals, b, op)
    assert x.shape == (2, bt.n)
    (0.5 * (x ** 2).sum()).backward()
    assert b.grad.shape == b.shape and vals.grad.shape == vals.shape
    # per batch: dL/db_k = A_k^{-T} x_k, summed over the batches
    gb = np.zeros(bt.n)
    for k, scale in enumerate((1.0, 1.5)):
        for s in range(bt.n_sys):
            r0, r1 = bt.row_off[s], bt.row_off[s + 1]
            A, _, _ = _dense(bt, s)
            xk = np.linalg.solve(scale * A, bt.b[r0:r1].astype(np.float64))
            gb[r0:r1] += np.linalg.solve(scale * A.T, xk)
    assert np.allclose(b.grad.cpu().numpy(), gb, rtol=1e-8, atol=1e-12)
    # interleaved forwards
    va = torch.from_numpy(v0).to(cuda).requires_grad_(True)
    vb = torch.from_numpy(2.0 * v0).to(cuda).requires_grad_(True)
    bb = torch.from_numpy(bt.b.astype(np.float64)).to(cuda)
    xa = sparse_solve(va, bb, op)
    xb = sparse_solve(vb, bb, op)
    (0.5 * (xa ** 2).sum()).backward()
    (0.5 * (xb ** 2).sum()).backward()
    # A x = b with A scaled by 2: x halves, dL/dA = -lambda x^T with lambda = A^-T x
    # scales by 1/8; the two gradients keep that ratio only if each backward
    # used its own forward's values
    assert np.allclose(vb.grad.cpu().numpy(), va.grad.cpu().numpy() / 8.0, rtol=1e-7, atol=1e-14)
