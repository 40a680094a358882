"""Systems whose rows are split over ranks (the multi-rank PaScaL_TDMA
path): the oracle's modified Thomas / reduced system / update against a
direct solve, and the exchange of pascal_poisson_fft_b200.dist on two and
four gloo ranks (CPU processes) with the oracle's per-rank steps."""
import os
import sys

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _systems(rng, n_row, n_sys):
    a = rng.uniform(-1, 1, (n_row, n_sys))
    c = rng.uniform(-1, 1, (n_row, n_sys))
    b = 2.5 + np.abs(a) + np.abs(c) + rng.uniform(0, 1, (n_row, n_sys))
    a[0] = 0.0
    c[-1] = 0.0
    d = rng.standard_normal((n_row, n_sys))
    return a, b, c, d


def split_solve_numpy(a, b, c, d, nranks):
    """The multi-rank algorithm with every rank emulated in one process."""
    rows = np.array_split(np.arange(d.shape[0]), nranks)
    parts = [[x[r].copy() for x in (a, b, c, d)] for r in rows]
    red = [O.tdma_modified(*p) for p in parts]
    n_sys = d.shape[1]
    ra = np.concatenate([r[0] for r in red])      # rank-major: 2 rows per rank
    rc = np.concatenate([r[1] for r in red])
    rd = np.concatenate([r[2] for r in red])
    O.tdma_many(ra, np.ones_like(ra), rc, rd)
    out = []
    for k, p in enumerate(parts):
        O.tdma_update(p[0], p[2], p[3], rd[2 * k:2 * k + 2])
        out.append(p[3])
    return np.concatenate(out)


@pytest.mark.parametrize("nranks,n_row", [(2, 16), (4, 64), (3, 40), (8, 24)])
def test_split_algorithm_matches_direct(nranks, n_row):
    rng = np.random.default_rng(nranks * 100 + n_row)
    a, b, c, d = _systems(rng, n_row, 37)
    x = split_solve_numpy(a, b, c, d, nranks)
    ref = d.copy()
    O.tdma_many(a.copy(), b.copy(), c.copy(), ref)
    assert np.linalg.norm(x - ref) <= 1e-13 * np.linalg.norm(ref)


class _OracleKernels:
    """Per-rank steps in the oracle, for CPU gloo ranks."""

    @staticmethod
    def modified(a, b, c, d, a_rd, c_rd, d_rd):
        ra, rc, rd = O.tdma_modified(a.numpy(), b.numpy(), c.numpy(), d.numpy())
        a_rd.numpy()[:] = ra
        c_rd.numpy()[:] = rc
        d_rd.numpy()[:] = rd

    @staticmethod
    def solve(a, b, c, d):
        O.tdma_many(a.numpy(), b.numpy(), c.numpy(), d.numpy())

    @staticmethod
    def update(a, c, d, x_rd):
        O.tdma_update(a.numpy(), c.numpy(), d.numpy(), x_rd.numpy())


def _worker(rank, ws, port, n_row, n_sys, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from pascal_poisson_fft_b200 import dist as D
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        rng = np.random.default_rng(42)
        a, b, c, d = _systems(rng, n_row, n_sys)
        rows = np.array_split(np.arange(n_row), ws)[rank]
        loc = [torch.from_numpy(np.ascontiguousarray(x[rows])) for x in (a, b, c, d)]
        D.tdma_many_dist(*loc, kernels=_OracleKernels)
        out.put((rank, rows.tolist(), loc[3].numpy().copy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ws", [2, 4])
def test_gloo_ranks_match_direct_solve(ws):
    import torch.multiprocessing as mp
    n_row, n_sys = 48, 29
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + ws + (os.getpid() % 1000)
    procs = [ctx.Process(target=_worker, args=(r, ws, port, n_row, n_sys, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=120) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    x = np.concatenate([r[2] for r in res])
    a, b, c, d = _systems(np.random.default_rng(42), n_row, n_sys)
    ref = d.copy()
    O.tdma_many(a, b, c, ref)
    assert np.linalg.norm(x - ref) <= 1e-13 * np.linalg.norm(ref)
    # and bit for bit the one-process emulation of the same algorithm
    a, b, c, d = _systems(np.random.default_rng(42), n_row, n_sys)
    assert np.array_equal(x, split_solve_numpy(a, b, c, d, ws))


def _halo_worker(rank, ws, port, periodic, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from pascal_poisson_fft_b200 import dist as D
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        rows = 3 + rank
        P = torch.full((rows + 2, 4, 5), -1.0, dtype=torch.float64)
        for k in range(1, rows + 1):
            P[k] = 100.0 * rank + k
        D.halo_exchange(P, rank, ws, periodic)
        out.put((rank, float(P[0, 0, 0]), float(P[rows + 1, 0, 0])))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ws,periodic", [(2, False), (2, True), (3, True), (3, False), (1, True)])
def test_gloo_halo_exchange(ws, periodic):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29800 + ws * 7 + int(periodic) + (os.getpid() % 500)
    procs = [ctx.Process(target=_halo_worker, args=(r, ws, port, periodic, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=120) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, lo, hi in res:
        below = rank - 1 if rank > 0 else (ws - 1 if periodic else None)
        above = rank + 1 if rank < ws - 1 else (0 if periodic else None)
        # lower ghost plane = last interior plane of the rank below, upper = first of the rank above
        assert lo == (100.0 * below + 3 + below if below is not None else -1.0)
        assert hi == (100.0 * above + 1 if above is not None else -1.0)
