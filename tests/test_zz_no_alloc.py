"""cmcg_dot_noalloc: the batched dot product for callers that must not let the
library allocate device memory (their own pool or framework allocator owns the
memory, or allocation is not allowed inside their loop). It must give the same
sums as cmcg_dot, call after call, using its fixed scratch array instead of an
allocation. Collected last so that a failure here comes after every other test."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


@pytest.mark.parametrize("dt,code,tol", [(torch.float64, 1, 1e-12), (torch.float32, 0, 2e-5)])
def test_dot_noalloc_matches_dot_twice(cuda, dt, code, tol):
    import cumat_b200 as cm
    from cumat_b200 import _native as N
    ctx = cm.Context.current()
    rng = np.random.default_rng(11)
    for n, batches in [(100003, 3), (7, 1), (4096, 1024)]:
        a = rng.uniform(-1, 1, (batches, n))
        b = rng.uniform(-1, 1, (batches, n))
        x = torch.from_numpy(a).to(dt).to(cuda)
        y = torch.from_numpy(b).to(dt).to(cuda)
        ref = torch.empty(batches, dtype=dt, device=cuda)
        N.call("cmcg_dot", ctx.handle, code, n, _ptr(x), batches, _ptr(y), batches, _ptr(ref))
        scale = (np.abs(a) * np.abs(b)).sum(1)
        for _ in range(2):   # two calls in a row share (and must reset) the scratch
            got = torch.full((batches,), float("nan"), dtype=dt, device=cuda)
            N.call("cmcg_dot_noalloc", ctx.handle, code, n, _ptr(x), batches, _ptr(y), batches, _ptr(got))
            g = got.cpu().double().numpy()
            r = ref.cpu().double().numpy()
            assert np.all(np.abs(g - r) <= tol * scale + 1e-300)


def test_dot_noalloc_rejects_too_many_batches(cuda):
    import cumat_b200 as cm
    from cumat_b200 import _native as N
    ctx = cm.Context.current()
    x = torch.ones((1025, 4), dtype=torch.float64, device=cuda)
    out = torch.empty(1025, dtype=torch.float64, device=cuda)
    with pytest.raises(cm.CuMatError, match="at most 1024"):
        N.call("cmcg_dot_noalloc", ctx.handle, 1, 4, _ptr(x), 1025, _ptr(x), 1025, _ptr(out))
