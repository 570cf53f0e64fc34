"""Multi-process (N > 1) plumbing of bench.py on CPU with the gloo backend,
world size 2: each rank gets its own batch (seed 2 + rank, no data exchange),
the step time is the maximum over ranks and the whole-job rate counts every
rank's systems. No GPU is involved."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        from cumat_b200 import problems as P
        seed = bench.rank_seed(rank)
        bt = P.fv2d_batch(8, bench.SIDE_LO, 32, bench.SIGMA, seed)
        local_ms = 10.0 + 5.0 * rank          # pretend device time of this rank
        ms = bench.max_over_ranks(world, local_ms)
        rate = bench.whole_job_rate(8, world, ms)
        out[rank] = (seed, int(bt.n), ms, rate)
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_and_timing():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        assert all(p.exitcode == 0 for p in procs)
        res = dict(out)
    assert res[0][0] != res[1][0]                      # different batches per rank
    assert res[0][2] == res[1][2] == 15.0              # max over ranks
    assert res[0][3] == pytest.approx(16 / 0.015)      # all ranks' systems / slowest time
