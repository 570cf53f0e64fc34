"""Batched reductions along any set of axes through the C ABI (cmcg_reduce):
the reference's known answers (tests/TestReductionOps2.cu, TestReductionOps3.cu)
and every axis combination, operation and kernel against numpy in FP64."""
import itertools
import json
from pathlib import Path

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

KAT = json.loads((Path(__file__).resolve().parent / "golden" / "reference_kats.json").read_text())
AXES = {"row": "rows", "column": "cols", "batch": "batches"}


def cm():
    import cumat_b200
    return cumat_b200


def _dev(data_brc, cuda, dt=torch.float64):
    # data[batch][row][col] -> memory [batch][col][row] (rows fastest)
    a = np.asarray(data_brc, np.float64).transpose(0, 2, 1)
    return torch.from_numpy(np.ascontiguousarray(a)).to(device=cuda, dtype=dt)


def _to_brc(out):
    return out.cpu().numpy().transpose(0, 2, 1)


@pytest.mark.parametrize("case", ["none", "column", "row", "batch", "row+column", "column+batch", "row+batch",
                                  "row+column+batch"])
@pytest.mark.parametrize("dt", [torch.float32, torch.float64])
def test_kat_axis_sums(cuda, case, dt):
    m = cm()
    k = KAT["reduce_axes"]
    axes = () if case == "none" else tuple(AXES[a] for a in case.split("+"))
    out = m.reduce(_dev(k["data"], cuda, dt), "sum", axes)
    assert np.array_equal(_to_brc(out), np.array(k["sum"][case], np.float64))


def test_kat_min_max_prod(cuda):
    m = cm()
    k = KAT["reduce_axes"]
    x = _dev(k["data"], cuda)
    allax = ("rows", "cols", "batches")
    assert float(m.reduce(x, "min", allax).item()) == k["min_all"]
    assert float(m.reduce(x, "max", allax).item()) == k["max_all"]
    kp = KAT["reduce_prod"]
    assert float(m.reduce(_dev(kp["data"], cuda), "prod", allax).item()) == kp["prod_all"]


def _numpy_reduce(a, op, axes):
    ax = tuple({"batches": 0, "cols": 1, "rows": 2}[n] for n in axes)
    f = {"sum": np.sum, "prod": np.prod, "min": np.min, "max": np.max}[op]
    return f(a, axis=ax, keepdims=True) if ax else a


SHAPES = [(1000, 3, 7), (5, 900, 4), (300, 200, 2), (100000, 2, 3), (7, 5, 3000), (1 << 20, 1, 1), (130, 1000, 3),
          (2, 3, 5000)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("kernel", [None, "thread", "warp", "block", "split", "tile"])
def test_all_axis_sets_vs_numpy(cuda, monkeypatch, shape, kernel):
    # every axis set (the tuned kernel, then each kernel forced where it
    # applies), sum / min / max in FP64 and FP32
    m = cm()
    if kernel:
        monkeypatch.setenv("CUMAT_REDUCE_KERNEL", kernel)
    R, Cc, B = shape
    rng = np.random.default_rng(R + Cc + B)
    a = rng.uniform(-1.0, 1.0, (B, Cc, R))
    for axes in itertools.chain.from_iterable(itertools.combinations(("rows", "cols", "batches"), k) for k in range(4)):
        ref_abs = _numpy_reduce(np.abs(a), "sum", axes)
        # FP32: the exact sum of the rounded inputs, within 2e-5 of the sum of
        # magnitudes (a serial FP32 sum of 2^20 terms included)
        for dt, tol in ((torch.float64, 1e-13), (torch.float32, 2e-5)):
            x = torch.from_numpy(a).to(device=cuda, dtype=dt)
            a_in = a.astype(np.float32).astype(np.float64) if dt == torch.float32 else a
            for op in ("sum", "min", "max"):
                got = m.reduce(x, op, axes).cpu().numpy().astype(np.float64)
                ref = _numpy_reduce(a_in, op, axes)
                assert got.shape == ref.shape
                if op == "sum":
                    assert np.all(np.abs(got - ref) <= tol * np.maximum(ref_abs, 1e-30) + 1e-30), (axes, dt, op)
                else:
                    assert np.array_equal(got, ref), (axes, dt, op)


def test_prod_and_log_callback(cuda):
    m = cm()
    msgs = []
    m.set_log_callback(lambda level, msg: msgs.append((level, msg)), 2)
    try:
        rng = np.random.default_rng(3)
        a = rng.uniform(0.9, 1.1, (3, 40, 50))
        x = torch.from_numpy(a).to(cuda)
        got = m.reduce(x, "prod", ("rows",)).cpu().numpy()
        assert np.allclose(got, np.prod(a, axis=2, keepdims=True), rtol=1e-12)
        # an invalid call reports its error through the hook too
        with pytest.raises(m.CuMatError):
            m._native.call("cmcg_reduce", m.Context.current().handle, 0, 9, 1, 1, 1, 1, None, None)
    finally:
        m.set_log_callback(None)
    assert any(level == 0 and "NULL" in msg for level, msg in msgs), msgs


@pytest.mark.parametrize("kernel", ["warp", "tile", "block", "split"])
@pytest.mark.parametrize("dt", [torch.float32, torch.float64])
def test_unaligned_input_takes_scalar_loads(cuda, monkeypatch, kernel, dt):
    # an input that starts 4 or 8 bytes past a 16-byte boundary (a slice of a
    # larger buffer): the warp and tile kernels step back to scalar loads,
    # block and split read each contiguous run with scalar loads up to the
    # first 16-byte boundary; same sums as numpy
    m = cm()
    monkeypatch.setenv("CUMAT_REDUCE_KERNEL", kernel)
    B, Cc, R = 3, 64, 256
    rng = np.random.default_rng(11)
    a = rng.uniform(-1.0, 1.0, (B, Cc, R))
    base = torch.zeros(B * Cc * R + 1, dtype=dt, device=cuda)
    base[1:] = torch.from_numpy(a.reshape(-1)).to(device=cuda, dtype=dt)
    x = base[1:].view(B, Cc, R)
    assert x.data_ptr() % 16 != 0
    a_in = a.astype(np.float32).astype(np.float64) if dt == torch.float32 else a
    tol = 2e-5 if dt == torch.float32 else 1e-13
    for axes in (("rows",), ("cols",), ("batches",), ("cols", "batches"), ("rows", "batches"), ("rows", "cols"),
                 ("rows", "cols", "batches")):
        got = m.reduce(x, "sum", axes).cpu().numpy().astype(np.float64)
        ref = _numpy_reduce(a_in, "sum", axes)
        scale = _numpy_reduce(np.abs(a), "sum", axes)
        assert np.all(np.abs(got - ref) <= tol * scale), (kernel, axes)
        for op in ("min", "max"):
            assert np.array_equal(m.reduce(x, op, axes).cpu().numpy().astype(np.float64), _numpy_reduce(a_in, op, axes))
