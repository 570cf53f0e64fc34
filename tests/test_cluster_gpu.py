"""The cluster solve of the grid path: systems of 16,385 .. 131,072 rows (FP32
vectors; 65,536 with FP64) solved by one thread-block cluster each, p / q / r /
x / 1/diag in the cluster's shared memory, scalars summed across the cluster's
CTAs, the values read in the diagonal layout (stencils) or the sliced layout.
Compared with the oracle's CG (reference cuMat/src/ConjugateGradient.h:123-206:
iteration counts within +-2, the same statuses) and with the graph loop of the
grid path on the same inputs."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from cumat_b200 import problems as P  # noqa: E402
from oracle import oracle as O  # noqa: E402


def cm():
    import cumat_b200
    return cumat_b200


def _csr(m, pr, dtype=torch.float32, systems=False, fmt="csr"):
    if fmt == "csr":
        p = m.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)
        vals = pr.val
    else:
        idx, vals = P.csr_to_ell(pr.n, pr.row_ptr, pr.col, pr.val)
        p = m.SparsityPattern.ell(pr.n, pr.n, idx)
    if systems:
        p.set_systems(pr.row_off)
    return m.SparseMatrix(p, dtype=dtype).setData(vals if dtype != torch.float64 else vals.astype(np.float64))


def _graph_solve(m, monkeypatch, A, b, tol, guess=None, max_iter=-1):
    monkeypatch.setenv("CUMAT_CG_CLUSTER", "0")
    monkeypatch.setenv("CUMAT_CG_COOP", "0")
    cg = m.ConjugateGradient(A).setTolerance(tol).setMaxIterations(max_iter).set_path(2)
    x = cg.solveWithGuess(b, guess) if guess is not None else cg.solve(b)
    monkeypatch.delenv("CUMAT_CG_CLUSTER")
    monkeypatch.delenv("CUMAT_CG_COOP")
    return x.cpu().numpy(), cg.system_stats()


@pytest.mark.parametrize("fmt", ["csr", "csr_sliced", "ell"])
def test_cluster_fp32_poisson_vs_oracle_and_graph(cuda, monkeypatch, fmt):
    # 2D Poisson 200^2 (40,000 rows: clusters of 10 CTAs x 4096 rows), FP32
    # Jacobi-CG to 1e-6: one cluster launch + the finaliser; the CSR pattern
    # is read in the diagonal layout, or (CUMAT_CG_DIA=0) the sliced layout
    m = cm()
    if fmt == "csr_sliced":
        monkeypatch.setenv("CUMAT_CG_DIA", "0")
    pr = P.poisson2d(200, 1)
    A = _csr(m, pr, fmt="ell" if fmt == "ell" else "csr")
    b = torch.from_numpy(pr.b).to(cuda)
    cg = m.ConjugateGradient(A).setTolerance(1e-6)
    cg.solve(b)
    before = m.launch_count()
    x = cg.solve(b).cpu().numpy()
    assert m.launch_count() - before == 2
    st = cg.system_stats()
    assert st["status"][0] == 0 and cg.error() < 1e-6
    _, it_o, _ = O.cg_csr(pr.n, pr.row_ptr, pr.col, pr.val, pr.b, 1e-6, -1, 1)
    assert abs(int(st["iterations"][0]) - int(it_o[0])) <= 2
    xg, sg = _graph_solve(m, monkeypatch, A, b, 1e-6)
    assert abs(int(sg["iterations"][0]) - int(st["iterations"][0])) <= 2
    assert np.linalg.norm(x - xg) / np.linalg.norm(xg) < 1e-4
    # deterministic: every CTA adds the partials in the same order
    assert np.array_equal(cg.solve(b).cpu().numpy(), x)
    assert m.Context.current().device_errors() == 0


def test_cluster_fp64_3d_vs_oracle(cuda, monkeypatch):
    # 3D 7-point FV system on 40^3 (64,000 rows: 16 CTAs x 4096 rows), FP64 to
    # 1e-10: iterations against the oracle, solution against the graph loop
    m = cm()
    p3 = P.fv3d(40, 1.0, 5)
    A = _csr(m, p3, dtype=torch.float64)
    b64 = p3.b.astype(np.float64)
    b = torch.from_numpy(b64).to(cuda)
    cg = m.ConjugateGradient(A).setTolerance(1e-10)
    x = cg.solve(b).cpu().numpy()
    st = cg.system_stats()
    assert st["status"][0] == 0 and cg.error() < 1e-10
    _, it_o, _ = O.cg_csr(p3.n, p3.row_ptr, p3.col, p3.val.astype(np.float64), b64, 1e-10, -1, 1)
    assert abs(int(st["iterations"][0]) - int(it_o[0])) <= 2
    xg, sg = _graph_solve(m, monkeypatch, A, b, 1e-10)
    assert np.linalg.norm(x - xg) / np.linalg.norm(xg) < 1e-9
    r = b64 - O.spmv_csr(p3.n, p3.n, p3.row_ptr, p3.col, p3.val.astype(np.float64), x)[0]
    assert np.linalg.norm(r) / np.linalg.norm(b64) < 2e-10


def test_cluster_packed_batches_vs_oracle(cuda):
    # three uneven systems of 17,161 .. 29,929 rows, two value batches (x1 and
    # x2): six instances, one cluster each, every system against the oracle
    m = cm()
    bt = P.fv2d_batch(3, 131, 173, 0.5, 31)
    p = m.SparsityPattern.csr(bt.n, bt.n, bt.row_ptr, bt.col)
    p.set_systems(bt.row_off)
    assert np.diff(bt.row_off).min() > 16384
    vals = np.stack([bt.val, 2.0 * bt.val]).astype(np.float32)
    A = m.SparseMatrix(p, dtype=torch.float32, batches=2).setData(vals)
    b = torch.from_numpy(np.tile(bt.b, 2)).to(cuda)
    cg = m.ConjugateGradient(A).setTolerance(1e-6)
    x = cg.solve(b.reshape(2, -1)).cpu().numpy().reshape(2, -1)
    st = cg.system_stats()
    assert st["status"].shape == (6,) and np.all(st["status"] == 0)
    for k in range(2):
        xo, it_o, _ = O.cg_packed(bt.row_off, bt.row_ptr, bt.col, vals[k], bt.b, 1e-6)
        its = st["iterations"][k * 3:(k + 1) * 3]
        assert np.all(np.abs(its.astype(np.int64) - it_o) <= 2), (its, it_o)
        assert np.linalg.norm(x[k] - xo) / np.linalg.norm(xo) < 1e-4
    # the second batch's matrix is twice the first: half the solution
    assert np.allclose(x[1], x[0] / 2, rtol=1e-3, atol=1e-6)


def test_cluster_guess_cap_zero_rhs_identity(cuda, monkeypatch):
    m = cm()
    pr = P.poisson2d(180, 2)
    A = _csr(m, pr)
    b = torch.from_numpy(pr.b).to(cuda)
    # an initial guess: the same solve as the graph loop from the same guess
    g = torch.from_numpy(np.random.default_rng(3).uniform(-1, 1, pr.n).astype(np.float32)).to(cuda)
    cg = m.ConjugateGradient(A).setTolerance(1e-6)
    x = cg.solveWithGuess(b, g).cpu().numpy()
    st = cg.system_stats()
    _, it_o, _ = O.cg_csr(pr.n, pr.row_ptr, pr.col, pr.val, pr.b, 1e-6, -1, 1, guess=g.cpu().numpy())
    assert st["status"][0] == 0 and abs(int(st["iterations"][0]) - int(it_o[0])) <= 2
    xg, _ = _graph_solve(m, monkeypatch, A, b, 1e-6, guess=g)
    assert np.linalg.norm(x - xg) / np.linalg.norm(xg) < 1e-4
    # iteration cap: MAX_ITER after exactly the cap
    cg2 = m.ConjugateGradient(A).setTolerance(1e-12).setMaxIterations(17)
    cg2.solve(b)
    s2 = cg2.system_stats()
    assert s2["status"][0] == m._native.SOLVE_MAX_ITER and int(s2["iterations"][0]) == 17
    # zero right-hand side: x = 0, ZERO_RHS
    cg3 = m.ConjugateGradient(A).setTolerance(1e-6)
    x3 = cg3.solve(torch.zeros_like(b)).cpu().numpy()
    assert cg3.system_stats()["status"][0] == m._native.SOLVE_ZERO_RHS and not np.any(x3)
    # identity preconditioner against the oracle
    cg4 = m.ConjugateGradient(A, m.IdentityPreconditioner).setTolerance(1e-6)
    cg4.solve(b)
    _, it_i, _ = O.cg_csr(pr.n, pr.row_ptr, pr.col, pr.val, pr.b, 1e-6, -1, 0)
    assert cg4.system_stats()["status"][0] == 0 and abs(cg4.iterations() - int(it_i[0])) <= 2
    assert m.Context.current().device_errors() == 0


def test_few_small_systems_take_the_cluster(cuda, monkeypatch):
    # one 100^2 Poisson system (10,000 rows: 10 CTAs x 1024 rows): the
    # automatic path gives a few systems above 4096 rows to the cluster solve
    # (one launch + the finaliser) instead of one CTA each; same result as the
    # one-CTA solver within the FP32 recursion's rounding
    m = cm()
    pr = P.poisson2d(100, 4)
    A = _csr(m, pr)
    b = torch.from_numpy(pr.b).to(cuda)
    cg = m.ConjugateGradient(A).setTolerance(1e-6)
    cg.solve(b)
    before = m.launch_count()
    x = cg.solve(b).cpu().numpy()
    assert m.launch_count() - before == 2
    st = cg.system_stats()
    _, it_o, _ = O.cg_csr(pr.n, pr.row_ptr, pr.col, pr.val, pr.b, 1e-6, -1, 1)
    assert st["status"][0] == 0 and abs(int(st["iterations"][0]) - int(it_o[0])) <= 2
    monkeypatch.setenv("CUMAT_CG_CLUSTER", "0")
    cg1 = m.ConjugateGradient(A).setTolerance(1e-6)
    x1 = cg1.solve(b).cpu().numpy()
    assert np.linalg.norm(x - x1) / np.linalg.norm(x1) < 1e-4
