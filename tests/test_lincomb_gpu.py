"""Fused linear combination (the reference's linear-combination benchmark
expression `v0 * f0 + v1 * f1 + ...`, benchmarks/linear_combination/
Implementation_cuMat.cu:52-66) against a float64 numpy sum: 1..16 terms,
16-byte and element-wise paths, batches with broadcast, accumulate modes."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def cm():
    import cumat_b200
    return cumat_b200


@pytest.mark.parametrize("k", [1, 2, 3, 5, 8, 10, 16])
@pytest.mark.parametrize("n", [1_000_000, 1001])   # vector path / element-wise path
def test_lincomb_terms(cuda, k, n):
    m = cm()
    rng = np.random.default_rng(k * 7 + n % 13)
    vs = [rng.uniform(0, 1, n).astype(np.float32) for _ in range(k)]
    f = rng.uniform(-1, 1, k)
    out = m.linear_combination(f, [torch.from_numpy(v).to(cuda) for v in vs]).cpu().numpy()
    want = sum(np.float64(c) * v.astype(np.float64) for c, v in zip(f.astype(np.float32), vs))
    assert np.allclose(out, want, rtol=2e-6 * k, atol=2e-6 * k)


def test_lincomb_batched_modes_fp64(cuda):
    m = cm()
    rng = np.random.default_rng(3)
    n = 4096
    a = rng.standard_normal((3, n))
    b = rng.standard_normal(n)                      # broadcast over the 3 batches
    ta, tb = torch.from_numpy(a).to(cuda), torch.from_numpy(b).to(cuda)
    out = m.linear_combination([2.0, -0.5], [ta, tb])
    assert out.shape == (3, n)
    assert np.allclose(out.cpu().numpy(), 2.0 * a - 0.5 * b[None, :], rtol=1e-14, atol=1e-14)
    acc = torch.ones((3, n), dtype=torch.float64, device=cuda)
    m.linear_combination([1.0], [ta], out=acc, mode=1)          # ADD
    assert np.allclose(acc.cpu().numpy(), 1.0 + a, rtol=1e-15, atol=1e-15)
    m.linear_combination([1.0], [ta], out=acc, mode=2)          # SUB
    assert np.allclose(acc.cpu().numpy(), 1.0, rtol=0, atol=1e-15)


def test_lincomb_rejects_bad_arguments(cuda):
    m = cm()
    v = torch.zeros(8, device=cuda)
    with pytest.raises(ValueError):
        m.linear_combination([1.0] * 17, [v] * 17)
    with pytest.raises(m.CuMatError):
        m.linear_combination([1.0, 1.0], [torch.zeros((2, 8), device=cuda), torch.zeros((3, 8), device=cuda)])
