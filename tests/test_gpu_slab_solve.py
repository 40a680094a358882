"""SlabPoisson.solve as a user calls it: one process per rank, a gloo
process group (every exchange staged through host memory), all ranks on the
one GPU.  No kernel waits on another rank's kernels (the exchanges are host
collectives between launches), so ranks sharing a GPU is safe.  The ghosted
slabs, gathered in rank 0, are compared with the single-GPU solve and the
oracle."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, ws, port, shape, pbc, beta, seed, out):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from pascal_poisson_fft_b200 import dist as D
    from pascal_poisson_fft_b200 import workloads as W
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=120))
    try:
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        p = W.random_problem(np.random.default_rng(seed), *shape, pbc, beta=beta)
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
        m = p.metrics
        slab = D.SlabPoisson(p.n1m, p.n2m, p.n3m, p.L1, p.L2, p.pbc, rank, ws, dev)
        P = torch.zeros(slab.ghost_shape(), dtype=torch.float64, device=dev)
        slab.solve(t(p.f[slab.z0:slab.z0 + slab.rows]), P, t(m["dmx1"]), t(m["dmx2"]), t(m["dmx3"]), t(m["dx3"]))
        torch.cuda.synchronize()
        out.put((rank, slab.z0, slab.rows, P.cpu().numpy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ws,shape,pbc", [(2, (64, 48, 40), (1, 1, 0)), (4, (48, 32, 33), (0, 0, 0)),
                                          (2, (32, 32, 32), (1, 1, 1)), (3, (40, 32, 24), (0, 1, 1))])
def test_slab_solve_on_gloo_ranks(ws, shape, pbc):
    import torch.multiprocessing as mp
    from _util import gpu_solve, oracle_solve, rel_l2
    from pascal_poisson_fft_b200 import workloads as W
    beta = 0.0 if pbc[2] else 1.5
    seed = sum(shape) + ws
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29900 + 11 * ws + sum(pbc) + (os.getpid() % 400)
    procs = [ctx.Process(target=_rank, args=(r, ws, port, shape, pbc, beta, seed, q)) for r in range(ws)]
    for pr in procs:
        pr.start()
    res = sorted((q.get(timeout=300) for _ in procs), key=lambda r: r[0])
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    p = W.random_problem(np.random.default_rng(seed), *shape, pbc, beta=beta)
    full = np.zeros((p.n3m + 2, p.n2m + 2, p.n1m + 2))
    full[0] = res[0][3][0]
    for _, z0, rows, P in res:
        full[1 + z0:1 + z0 + rows] = P[1:rows + 1]
    full[p.n3m + 1] = res[-1][3][res[-1][2] + 1]
    # every rank's lower and upper ghost plane is its neighbour's boundary plane
    for k, (_, z0, rows, P) in enumerate(res):
        assert np.array_equal(P[1:rows + 1], full[1 + z0:1 + z0 + rows])
        if k > 0 or pbc[2]:
            assert np.allclose(P[0], full[z0] if k > 0 else full[p.n3m], rtol=0, atol=0)
        if k < ws - 1 or pbc[2]:
            assert np.allclose(P[rows + 1], full[z0 + rows + 1] if k < ws - 1 else full[1], rtol=0, atol=0)
    # the modified Thomas eliminates in another order than Thomas: the
    # ill-conditioned low modes agree to cond * eps, not bit for bit
    assert rel_l2(full, gpu_solve(p)) < 1e-10
    assert rel_l2(full, oracle_solve(p)) < 1e-10
