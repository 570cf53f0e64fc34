"""Every device-side wait of the library is bounded and reports that it ran out.

Two waits exist: the grid barrier of the cooperative one-launch CG (a CTA
polls a release word the last arriving CTA writes) and the stage barriers of
the bulk-copy CSR product (threads wait for the copies of a tile to land). The
tests make each wait run out without faulting or hanging anything: the
library reads a short limit from the environment at launch time, and

* the grid barrier is told to expect one arrival more than the CTAs of the
  launch, so no CTA is ever the last and every poll runs out;
* the product's stages are armed (expected bytes posted) but no copy is
  issued, so no asynchronous copy is in flight when the wait gives up.

Each test checks that the call returns, that the context's device error word
carries the matching bit (1 = stage barrier, 2 = grid barrier), that the
solve is not reported converged, and that the context still works
afterwards."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from cumat_b200 import problems as P  # noqa: E402
from oracle import oracle as O  # noqa: E402


def cm():
    import cumat_b200
    return cumat_b200


def test_grid_barrier_wait_runs_out(cuda, monkeypatch):
    m = cm()
    pr = P.poisson2d(64, 0)
    A = m.SparseMatrix(m.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(pr.val)
    b = torch.from_numpy(pr.b).to(cuda)
    ctx = m.Context.current()
    ctx.device_errors()   # clear
    monkeypatch.setenv("CUMAT_TEST_GRID_SPINS", "2000")
    monkeypatch.setenv("CUMAT_TEST_GRID_EXTRA", "1")
    cg = m.ConjugateGradient(A).setTolerance(1e-6).set_path(2)   # one system: the cooperative launch
    cg.solve(b)
    flags = ctx.device_errors()
    assert flags & 2, flags
    st = cg.system_stats()
    assert st["status"][0] != 0   # not converged
    # the same solve with the normal limit converges on the same context
    monkeypatch.delenv("CUMAT_TEST_GRID_SPINS")
    monkeypatch.delenv("CUMAT_TEST_GRID_EXTRA")
    cg2 = m.ConjugateGradient(A).setTolerance(1e-6).set_path(2)
    x = cg2.solve(b).cpu().numpy()
    assert ctx.device_errors() == 0
    assert cg2.system_stats()["status"][0] == 0 and cg2.error() < 1e-6
    _, it_o, _ = O.cg_csr(pr.n, pr.row_ptr, pr.col, pr.val, pr.b, 1e-6, -1, 1)
    assert abs(cg2.iterations() - int(it_o[0])) <= 2
    assert np.all(np.isfinite(x))


def test_bulk_copy_stage_wait_runs_out(cuda, monkeypatch):
    m = cm()
    pr = P.poisson2d(256, 3)
    A = m.SparseMatrix(m.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(pr.val)
    x = torch.from_numpy(pr.b).to(cuda)
    ctx = m.Context.current()
    ctx.device_errors()
    monkeypatch.setenv("CUMAT_SPMV_VARIANT", "2")     # the bulk-copy CSR product
    monkeypatch.setenv("CUMAT_TEST_WAIT_LIMIT", "2000")
    monkeypatch.setenv("CUMAT_TEST_NO_COPY", "1")
    A * x
    flags = ctx.device_errors()
    assert flags & 1, flags
    # with copies and the normal limit the same kernel is correct again
    monkeypatch.delenv("CUMAT_TEST_WAIT_LIMIT")
    monkeypatch.delenv("CUMAT_TEST_NO_COPY")
    y = (A * x).cpu().numpy()
    assert ctx.device_errors() == 0
    ref = O.spmv_csr(pr.n, pr.n, pr.row_ptr, pr.col, pr.val, pr.b)[0]
    assert np.array_equal(y, ref)
