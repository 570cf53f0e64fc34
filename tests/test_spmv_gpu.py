"""SpMV, reductions and the sampled outer product through the C ABI on the GPU,
against the reference's known answers and the CPU oracle."""
import json
from pathlib import Path

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from cumat_b200 import problems as P  # noqa: E402
from oracle import oracle as O  # noqa: E402

KAT = json.loads((Path(__file__).resolve().parent / "golden" / "reference_kats.json").read_text())


def _cm():
    import cumat_b200 as cm
    return cm


def _csr_pattern(k):
    cm = _cm()
    return cm.SparsityPattern.csr(k["rows"], k["cols"], k["JA"], k["IA"])


def test_kat_csr_product(cuda):
    cm = _cm()
    k = KAT["spmv_csr"]
    A = cm.SparseMatrix(_csr_pattern(k)).setData(np.array(k["values"], np.float32))
    x = torch.tensor(k["x"], dtype=torch.float32, device=cuda)
    y0 = (A * x).cpu().tolist()                     # first product: kernel picked by timing
    before = cm.launch_count()
    y = A * x
    assert cm.launch_count() - before == 1          # one kernel per product afterwards
    assert y.cpu().tolist() == k["y"] == y0
    k2 = KAT["spmv_csr_scaled_matrix"]
    A2 = cm.SparseMatrix(_csr_pattern(k)).setData(np.array(k["values"], np.float32) * k2["scale"])
    assert (A2 * x).cpu().tolist() == k2["y"]


@pytest.mark.parametrize("case", ["spmv_csr_batched_matrix", "spmv_csr_batched_vector", "spmv_csr_batched_both"])
@pytest.mark.parametrize("dt", [torch.float32, torch.float64])
def test_kat_csr_batched(cuda, case, dt):
    cm = _cm()
    k = KAT[case]
    ms, vs = k.get("matrix_scales", [1]), k.get("vector_scales", [1])
    vals = np.stack([np.array(k["values"], np.float64) * s for s in ms])
    A = cm.SparseMatrix(_csr_pattern(k), dtype=dt, batches=len(ms)).setData(vals)
    X = torch.tensor(np.stack([np.array(k["x"], np.float64) * s for s in vs]), dtype=dt, device=cuda)
    y = A.product(X)
    expect = np.stack([np.array(k["y"], np.float64) * s for s in k["y_scales"]])
    assert np.array_equal(y.cpu().numpy(), expect)


@pytest.mark.parametrize("case", ["spmv_ell", "spmv_ell_batched_both"])
def test_kat_ell(cuda, case):
    cm = _cm()
    k = KAT[case]
    p = cm.SparsityPattern.ell(k["rows"], k["cols"], k["indices"])
    ms, vs = k.get("matrix_scales", [1]), k.get("vector_scales", [1])
    vals = np.stack([np.array(k["values"], np.float32) * s for s in ms])
    A = cm.SparseMatrix(p, batches=len(ms)).setData(vals)
    X = torch.tensor(np.stack([np.array(k["x"], np.float32) * s for s in vs]), device=cuda)
    y = A.product(X)
    expect = np.stack([np.array(k["y"], np.float32) * s for s in k.get("y_scales", [1])])
    assert np.array_equal(y.cpu().numpy().reshape(expect.shape), expect)
    # the pattern round-trips bit-exactly, padding -1 included
    assert np.array_equal(p.download(), np.array(k["indices"], np.int32))


def _random_csr(rng, rows, cols, max_len, empty_frac=0.1):
    lens = rng.integers(0, max_len + 1, rows)
    lens[rng.random(rows) < empty_frac] = 0
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(cols, l, replace=False)) for l in lens]).astype(np.int32) if lens.sum() else np.zeros(0, np.int32)
    return rp, ci


@pytest.mark.parametrize("max_len", [1, 5, 40, 300])
@pytest.mark.parametrize("mdt", [torch.float32, torch.float64, torch.bfloat16])
def test_random_csr_vs_oracle(cuda, max_len, mdt):
    cm = _cm()
    rng = np.random.default_rng(max_len)
    rows, cols = 777, 901
    rp, ci = _random_csr(rng, rows, cols, max_len)
    vals = rng.uniform(-1, 1, (2, ci.size)).astype(np.float32)
    if mdt == torch.bfloat16:
        vals = O.bf16_round(vals)
    A = cm.SparseMatrix(cm.SparsityPattern.csr(rows, cols, rp, ci), dtype=mdt, batches=2).setData(vals)
    for vdt, npdt, tol in [(torch.float32, np.float32, 1e-6), (torch.float64, np.float64, 1e-13)]:
        x = rng.uniform(-1, 1, (2, cols)).astype(npdt)
        y = A.product(torch.from_numpy(x).to(cuda)).cpu().numpy()
        ref = O.spmv_csr(rows, cols, rp, ci, vals.astype(np.float64), x.astype(np.float64))
        scale = O.spmv_csr(rows, cols, rp, ci, np.abs(vals).astype(np.float64), np.abs(x).astype(np.float64))
        assert np.all(np.abs(y - ref) <= tol * np.maximum(scale, 1e-30) + 1e-30)
        assert np.all(y[:, np.diff(rp) == 0] == 0)   # empty rows give 0


def test_assignment_modes(cuda):
    cm = _cm()
    k = KAT["spmv_csr"]
    A = cm.SparseMatrix(_csr_pattern(k)).setData(np.array(k["values"], np.float32))
    x = torch.tensor(k["x"], dtype=torch.float32, device=cuda)
    y = torch.ones(4, device=cuda)
    A.product(x, out=y, mode=1)
    assert y.cpu().tolist() == [v + 1 for v in k["y"]]
    A.product(x, out=y, mode=2)
    assert y.cpu().tolist() == [1.0] * 4


def test_poisson_1024_product_and_ell_agree(cuda):
    cm = _cm()
    pr = P.poisson2d(1024, 1)
    p = cm.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)
    A = cm.SparseMatrix(p).setData(pr.val)
    idx, ev = P.csr_to_ell(pr.n, pr.row_ptr, pr.col, pr.val)
    E = cm.SparseMatrix(cm.SparsityPattern.ell(pr.n, pr.n, idx)).setData(ev)
    x = torch.from_numpy(pr.b).to(cuda)
    y = A * x
    ye = E * x
    ref = O.spmv_csr(pr.n, pr.n, pr.row_ptr, pr.col, pr.val, pr.b)[0]
    assert np.array_equal(y.cpu().numpy(), ref)       # exact: integer-valued stencil, one rounding per row
    assert np.array_equal(ye.cpu().numpy(), ref)
    ja, ia = p.download()
    assert np.array_equal(ja, pr.row_ptr) and np.array_equal(ia, pr.col)
    assert np.array_equal(A.getData()[0], pr.val)


def test_kat_dot_norm(cuda):
    cm = _cm()
    k = KAT["dot"]
    x = torch.tensor(k["x"], dtype=torch.float64, device=cuda)
    y = torch.tensor(k["y"][0], dtype=torch.float64, device=cuda)
    assert cm.dot(x, y.unsqueeze(0)).cpu().tolist() == k["out"]
    assert cm.dot(y.unsqueeze(0), x).cpu().tolist() == k["out"]
    k = KAT["squared_norm"]
    x = torch.tensor(k["x"], dtype=torch.float64, device=cuda)
    assert cm.squaredNorm(x).cpu().tolist() == k["out"]
    assert np.allclose(cm.norm(x).cpu().numpy(), k["norm"], rtol=1e-15)


@pytest.mark.parametrize("n", [1, 10, 1000, 100000, 1000000, 10000001])
def test_large_reductions(cuda, n):
    cm = _cm()
    rng = np.random.default_rng(n)
    a = rng.uniform(-1, 1, (3, n))
    b = rng.uniform(-1, 1, (3, n))
    ref = (a * b).sum(1)
    for dt, tol in [(torch.float64, 1e-12), (torch.float32, 2e-5)]:
        xa = torch.from_numpy(a).to(dt).to(cuda)
        xb = torch.from_numpy(b).to(dt).to(cuda)
        got = cm.dot(xa, xb).cpu().double().numpy()
        scale = (np.abs(a) * np.abs(b)).sum(1)
        assert np.all(np.abs(got - ref) <= tol * scale + 1e-300)
        r1 = cm.dot(xa, xb).cpu().numpy()
        assert np.array_equal(r1, cm.dot(xa, xb).cpu().numpy())   # deterministic


def test_kat_outer_product_on_pattern(cuda):
    cm = _cm()
    k = KAT["outer_product_on_pattern"]
    p = cm.SparsityPattern.csr(k["rows"], k["cols"], k["JA"], k["IA"])
    A = cm.SparseMatrix(p, dtype=torch.float64)
    u = torch.tensor(k["u"], dtype=torch.float64, device=cuda)
    v = torch.tensor(k["v"], dtype=torch.float64, device=cuda)
    vals = cm.sddmm(A, u, v)[0].cpu().numpy()
    dense = np.zeros((5, 5))
    for r in range(5):
        for j in range(k["JA"][r], k["JA"][r + 1]):
            dense[r, k["IA"][j]] = vals[j]
    assert np.array_equal(dense, np.array(k["dense"]))


def test_sddmm_random_vs_oracle(cuda):
    cm = _cm()
    rng = np.random.default_rng(5)
    rp, ci = _random_csr(rng, 500, 600, 20)
    A = cm.SparseMatrix(cm.SparsityPattern.csr(500, 600, rp, ci), dtype=torch.float64)
    u = rng.standard_normal(500)
    v = rng.standard_normal(600)
    got = cm.sddmm(A, torch.from_numpy(u).to(cuda), torch.from_numpy(v).to(cuda), alpha=-1.0)[0].cpu().numpy()
    assert np.array_equal(got, O.sddmm_csr(500, rp, ci, u, v, alpha=-1.0))


def test_invalid_patterns_raise(cuda):
    cm = _cm()
    with pytest.raises(cm.CuMatError):
        cm.SparsityPattern.csr(2, 2, [0, 2, 1], [0, 1])        # decreasing row_ptr
    with pytest.raises(cm.CuMatError):
        cm.SparsityPattern.csr(2, 2, [0, 1, 2], [0, 2])        # column out of range
    with pytest.raises(cm.CuMatError):
        cm.SparsityPattern.ell(2, 2, [[0, -2], [1, 0]])        # bad padding index
    p = cm.SparsityPattern.csr(4, 4, [0, 1, 2, 3, 4], [0, 2, 1, 3])
    with pytest.raises(cm.CuMatError):
        p.set_systems([0, 2, 4])                                # (1, 2) couples two systems


@pytest.mark.parametrize("fmt", ["csr", "ell"])
def test_autotuned_product_is_deterministic(cuda, fmt):
    # the first product times the candidate kernels; they add every row in the
    # same order, so the tuned product gives the same bits as the first one
    cm = _cm()
    pr = P.poisson2d(300, 4)
    vals = (pr.val * P.uniform(5, pr.nnz, 0.5, 1.5)).astype(np.float32)
    if fmt == "csr":
        A = cm.SparseMatrix(cm.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(vals)
    else:
        idx, ev = P.csr_to_ell(pr.n, pr.row_ptr, pr.col, vals)
        A = cm.SparseMatrix(cm.SparsityPattern.ell(pr.n, pr.n, idx)).setData(ev)
    x = torch.from_numpy(pr.b).to(cuda)
    y1 = (A * x).cpu().numpy()
    y2 = (A * x).cpu().numpy()
    assert np.array_equal(y1, y2)
    yo = O.spmv_csr(pr.n, pr.n, pr.row_ptr, pr.col, vals, pr.b)[0]
    assert np.allclose(y1, yo, rtol=1e-6, atol=1e-6 * np.abs(yo).max())


def _row_abs_sums(rp, w):
    """Per-row sums of w over CSR rows (0 for empty rows)."""
    out = np.add.reduceat(np.append(w, 0.0), rp[:-1].astype(np.int64))
    out[np.diff(rp) == 0] = 0.0
    return out


def _power_law_csr(n, seed, alpha=1.1, scale=2.0, max_len=None):
    """Rows whose lengths follow a heavy-tailed (Pareto) law, sorted distinct
    random columns, values U[-1, 1]: the skewed case thread-per-row handles
    worst (a few rows hold thousands of entries)."""
    rng = np.random.default_rng(seed)
    max_len = max_len or n
    lens = np.minimum((rng.pareto(alpha, n) * scale + 1).astype(np.int64), max_len)
    rp = np.zeros(n + 1, np.int64)
    rp[1:] = np.cumsum(lens)
    col = np.empty(int(rp[-1]), np.int32)
    for r in range(n):
        col[rp[r]:rp[r + 1]] = np.sort(rng.choice(n, size=int(lens[r]), replace=False))
    val = rng.uniform(-1.0, 1.0, col.size)
    return rp.astype(np.int32), col, val


@pytest.mark.parametrize("dt", [torch.float32, torch.float64])
def test_power_law_csr_vs_oracle(cuda, dt):
    # the row-length rule gives this pattern the warp-per-row kernel (its
    # longest rows are far above 32 times the mean)
    cm = _cm()
    n = 20000
    rp, col, val = _power_law_csr(n, 5)
    lens = np.diff(rp)
    assert lens.max() >= 256 and lens.max() >= 32 * lens.mean()
    npdt = np.float32 if dt == torch.float32 else np.float64
    A = cm.SparseMatrix(cm.SparsityPattern.csr(n, n, rp, col), dtype=dt).setData(val.astype(npdt))
    xh = np.random.default_rng(6).uniform(-1.0, 1.0, n).astype(npdt)
    y = (A * torch.from_numpy(xh).to(cuda)).cpu().numpy()
    ref = O.spmv_csr(n, n, rp, col, val.astype(npdt), xh)[0].astype(np.float64)
    scale = _row_abs_sums(rp, np.abs(val) * np.abs(xh.astype(np.float64))[col])
    tol = 1e-6 if dt == torch.float32 else 1e-13
    # relative to the row's sum of |a_ij x_j| (the conditioning of each row sum)
    assert np.all(np.abs(y - ref) <= tol * np.maximum(scale, 1e-30)), np.max(np.abs(y - ref) / scale)


@pytest.mark.parametrize("variant", [3, 4, 5, 6])
def test_lanes_per_row_kernels_vs_oracle(cuda, monkeypatch, variant):
    # every V-lanes-per-row kernel (V = 4, 8, 16, 32), forced, on a random CSR
    # matrix with rows of 0..60 entries, batched values and vectors
    cm = _cm()
    monkeypatch.setenv("CUMAT_SPMV_VARIANT", str(variant))
    rng = np.random.default_rng(variant)
    n = 3000
    lens = rng.integers(0, 61, n)
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum(lens)
    col = np.concatenate([np.sort(rng.choice(n, size=int(k), replace=False)) for k in lens]).astype(np.int32)
    vals = rng.uniform(-1.0, 1.0, (2, col.size)).astype(np.float32)
    A = cm.SparseMatrix(cm.SparsityPattern.csr(n, n, rp, col), batches=2).setData(vals)
    X = rng.uniform(-1.0, 1.0, (2, n)).astype(np.float32)
    y = A.product(torch.from_numpy(X).to(cuda)).cpu().numpy()
    ref = O.spmv_csr(n, n, rp, col, vals, X)
    scale = np.stack([_row_abs_sums(rp, np.abs(vals[b]).astype(np.float64) * np.abs(X[b])[col]) for b in range(2)])
    scale[:, lens == 0] = 1.0
    assert np.all(np.abs(y - ref) <= 1e-6 * scale)
    assert np.all(y[:, lens == 0] == 0)


def test_tuning_cache_records_the_choice(cuda, monkeypatch, tmp_path):
    # a timed choice is written to the cache file and read back by a new
    # pattern of the same shape (no second timing: one launch per product)
    cm = _cm()
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("CUMAT_TUNE_CACHE", str(cache))
    pr = P.poisson2d(300, 2)
    A = cm.SparseMatrix(cm.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(pr.val)
    x = torch.from_numpy(pr.b).to(cuda)
    y0 = (A * x).cpu().numpy()
    lines = cache.read_text().split("\n")
    key = f"|csr|0|0|{pr.n}|{pr.nnz}|0 "
    assert any(key in (l + " ") and l.split()[-1] in ("0", "2", "7", "8", "9") for l in lines if l), lines
    B = cm.SparseMatrix(cm.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(pr.val)
    before = cm.launch_count()
    y1 = (B * x).cpu().numpy()
    assert cm.launch_count() - before == 1
    assert np.array_equal(y0, y1)


@pytest.mark.parametrize("dt", [torch.float32, torch.float64, torch.bfloat16])
@pytest.mark.parametrize("variant,max_len", [("7", 12), ("8", 12), ("8", 700), ("9", 12), ("9", 700)])
def test_row_order_kernels_equal_thread_per_row(cuda, monkeypatch, dt, variant, max_len):
    # the 16-byte-chunk kernel (variant 7), the warp-staged kernel (variant 8)
    # and thread per row with two rows in flight (variant 9) add every row in
    # entry order with fused multiply-adds, so they equal thread per row
    # (variant 0) bit for bit: random rows of 0..max_len
    # entries (empty rows, a row count that is not a multiple of 4 or 32, and
    # with max_len 700 rows that span several staging rounds of 256 entries),
    # two batches of values and vectors, all assignment modes
    cm = _cm()
    rng = np.random.default_rng(17 + max_len)
    n = 5003 if max_len < 100 else 701
    lens = rng.integers(0, max_len + 1, n)
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum(lens)
    col = np.concatenate([np.sort(rng.choice(n, size=int(k), replace=False)) for k in lens]).astype(np.int32)
    vals = rng.uniform(-1.0, 1.0, (2, col.size))
    A = cm.SparseMatrix(cm.SparsityPattern.csr(n, n, rp, col), dtype=dt, batches=2).setData(vals)
    vdt = torch.float64 if dt == torch.float64 else torch.float32
    X = torch.from_numpy(rng.uniform(-1.0, 1.0, (2, n))).to(device=cuda, dtype=vdt)
    out = {}
    for v in ("0", variant):
        monkeypatch.setenv("CUMAT_SPMV_VARIANT", v)
        res = [A.product(X).cpu().numpy()]
        for mode in (cm._native.ADD, cm._native.SUB):
            y = torch.ones((2, n), dtype=vdt, device=cuda)
            A.product(X, out=y, mode=mode)
            res.append(y.cpu().numpy())
        out[v] = res
    for a, b in zip(out["0"], out[variant]):
        assert np.array_equal(a, b)
    assert np.all(out[variant][0][:, lens == 0] == 0)
