"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (one process
each), the max-over-ranks step time, and the reference arm running on rank 0
only."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, ws, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        env = bench.dist_env()
        got = bench.max_over_ranks(1.5 + rank, ws)
        dist.barrier()
        # the reference arm returns at once, without work, on every rank but 0
        skipped = bench.run_reference(None, ws, rank) is None if rank != 0 else None
        out.put((rank, env, got, skipped))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_step():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 2000)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [(2, 0, 0), (2, 1, 1)]
    assert all(r[2] == pytest.approx(2.5) for r in res)
    assert res[1][3] is True
