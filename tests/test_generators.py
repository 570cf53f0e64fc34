"""Synthetic problem generators: bit-exact patterns, value rules, packing. CPU only."""
import numpy as np
import pytest

from cumat_b200 import problems as P


def _poisson_eigen_order(g):
    """Independent construction of the reference benchmark's matrix
    (benchmarks/conjugate_gradient/Implementation_cuMat.cu:29-41) as Eigen's
    RowMajor compressed storage (columns sorted within a row)."""
    rows, cols, vals = [], [], []
    idx = lambda x, y: y + x * g  # noqa: E731
    for x in range(g):
        for y in range(g):
            r = idx(x, y)
            ent = []
            if x > 0: ent.append((idx(x - 1, y), -1.0))
            if y > 0: ent.append((idx(x, y - 1), -1.0))
            ent.append((r, 4.0))
            if y < g - 1: ent.append((idx(x, y + 1), -1.0))
            if x < g - 1: ent.append((idx(x + 1, y), -1.0))
            ent.sort()
            for c, v in ent:
                rows.append(r); cols.append(c); vals.append(v)
    rp = np.zeros(g * g + 1, np.int64)
    np.add.at(rp, np.array(rows) + 1, 1)
    return np.cumsum(rp), np.array(cols), np.array(vals)


@pytest.mark.parametrize("g", [1, 2, 5, 64])
def test_poisson_pattern_bit_exact(g):
    pr = P.poisson2d(g, 0)
    rp, ci, v = _poisson_eigen_order(g)
    assert np.array_equal(pr.row_ptr, rp) and np.array_equal(pr.col, ci)
    assert np.array_equal(pr.val, v.astype(np.float32))
    assert pr.nnz == 5 * g * g - 4 * g


def test_config_sizes():
    assert P.poisson2d(64, 0).nnz == 20224
    assert P._L().cmgen_poisson2d_nnz(1024) == 5238784
    assert P._L().cmgen_fv3d_nnz(256) == 117047296


def test_uniform_rhs_is_mt19937():
    # std::mt19937(0) + uniform_real_distribution<float>(-1, 1): first draw of seed 0
    b = P.uniform(0, 3)
    assert b.dtype == np.float32 and np.all(np.abs(b) <= 1)
    assert np.array_equal(b, P.uniform(0, 3)) and not np.array_equal(b, P.uniform(1, 3))


def test_fv2d_kappa_one_is_poisson():
    bt = P.fv2d_batch(3, 7, 7, 0.0, 9)
    pr = P.poisson2d(7, 0)
    for s in range(3):
        rp, ci, v = bt.system(s)
        assert np.array_equal(rp, pr.row_ptr) and np.array_equal(ci, pr.col) and np.array_equal(v, pr.val)


def test_fv2d_batch_structure():
    bt = P.fv2d_batch(20, 4, 12, 0.5, 2)
    assert np.array_equal(np.diff(bt.row_off), bt.sides.astype(np.int64) ** 2)
    assert np.all((bt.sides >= 4) & (bt.sides <= 12))
    for s in range(bt.n_sys):
        rp, ci, v = bt.system(s)
        n = bt.row_off[s + 1] - bt.row_off[s]
        assert ci.min() >= 0 and ci.max() < n                     # block diagonal
        A = np.zeros((n, n))
        for r in range(n):
            A[r, ci[rp[r]:rp[r + 1]]] = v[rp[r]:rp[r + 1]]
            assert np.all(np.diff(ci[rp[r]:rp[r + 1]]) > 0)      # sorted columns
        assert np.allclose(A, A.T)                                 # symmetric
        assert np.all(np.linalg.eigvalsh(A) > 0)                   # SPD
        off = A - np.diag(np.diag(A))
        assert np.all(np.diag(A) >= -off.sum(1) * (1 - 1e-6))      # diagonally dominant
    # the batch of configuration 3 draws sides first: same sides for the dims query
    sides = np.empty(20, np.int32)
    import ctypes as C
    r, z = C.c_int64(), C.c_int64()
    P._L().cmgen_fv2d_batch_dims(20, 4, 12, 2, sides.ctypes.data_as(C.c_void_p), C.byref(r), C.byref(z))
    assert np.array_equal(sides, bt.sides) and r.value == bt.n and z.value == bt.nnz


def test_fv3d_structure():
    p = P.fv3d(5, 1.0, 3)
    assert p.n == 125 and p.nnz == 7 * 125 - 6 * 25
    A = np.zeros((p.n, p.n))
    for r in range(p.n):
        A[r, p.col[p.row_ptr[r]:p.row_ptr[r + 1]]] = p.val[p.row_ptr[r]:p.row_ptr[r + 1]]
    assert np.allclose(A, A.T) and np.all(np.linalg.eigvalsh(A) > 0)


def test_csr_to_ell_slot_order_and_padding():
    pr = P.poisson2d(4, 0)
    idx, val = P.csr_to_ell(pr.n, pr.row_ptr, pr.col, pr.val)
    assert idx.shape == (16, 5)
    # interior row: slots W, S, C, N, E
    r = 1 + 4 * 1
    assert list(idx[r]) == [r - 4, r - 1, r, r + 1, r + 4]
    # corner row 0: C, N, E then padding -1 / 0
    assert list(idx[0]) == [0, 1, 4, -1, -1] and list(val[0]) == [4, -1, -1, 0, 0]
