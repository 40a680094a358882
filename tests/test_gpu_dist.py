"""The multi-rank TDMA kernels on one GPU: every rank of the z-slab split
emulated in one process (each rank's kernels launched in turn, the
all-to-all done by stacking the ranks' send buffers), against the oracle's
emulation of the same algorithm (bit for bit) and the direct solve."""
import numpy as np
import pytest

from oracle import oracle as O
from test_dist_tdma import _systems, split_solve_numpy

pytestmark = pytest.mark.gpu


def _gpu_split_solve(a, b, c, d, nranks):
    import torch
    from pascal_poisson_fft_b200 import dist as D
    dev = torch.device("cuda", 0)
    rows = np.array_split(np.arange(d.shape[0]), nranks)
    n_sys = d.shape[1]
    loc = [[torch.as_tensor(np.ascontiguousarray(x[r]), device=dev) for x in (a, b, c, d)] for r in rows]
    sends = []
    for p in loc:
        a_rd, c_rd, d_rd = (torch.empty((2, n_sys), dtype=torch.float64, device=dev) for _ in range(3))
        D._Kernels.modified(*p, a_rd, c_rd, d_rd)
        sends.append(D.pack_reduced(a_rd, c_rd, d_rd, nranks))
    # all-to-all: rank k receives slice k of every rank's buffer
    backs = []
    for k in range(nranks):
        recv = torch.stack([s[k] for s in sends])
        ra, rb, rc, rd = D.reduced_systems(recv)
        D._Kernels.solve(ra, rb, rc, rd)
        backs.append(D.pack_solution(rd))
    out = []
    for k, p in enumerate(loc):
        recv = torch.stack([bk[k] for bk in backs])
        D._Kernels.update(p[0], p[2], p[3], D.unpack_solution(recv, n_sys))
        out.append(p[3])
    torch.cuda.synchronize()
    return torch.cat(out).cpu().numpy()


@pytest.mark.parametrize("nranks,n_row,n_sys", [(2, 16, 37), (4, 64, 1000), (8, 512, 4097), (3, 40, 130)])
def test_split_kernels_match_oracle(nranks, n_row, n_sys):
    rng = np.random.default_rng(nranks + n_row)
    a, b, c, d = _systems(rng, n_row, n_sys)
    x = _gpu_split_solve(a, b, c, d, nranks)
    assert np.array_equal(x, split_solve_numpy(a, b, c, d, nranks))
    ref = d.copy()
    O.tdma_many(a.copy(), b.copy(), c.copy(), ref)
    assert np.linalg.norm(x - ref) <= 1e-13 * np.linalg.norm(ref)


def test_rejects_short_slabs():
    import torch
    import pascal_poisson_fft_b200 as ppf
    from pascal_poisson_fft_b200 import dist as D
    t = [torch.ones((2, 8), dtype=torch.float64, device="cuda") for _ in range(4)]
    r = [torch.empty((2, 8), dtype=torch.float64, device="cuda") for _ in range(3)]
    with pytest.raises(ppf.PPFError):
        D._Kernels.modified(*t, *r)


def _emulated_slab_solve(p, nranks):
    """SlabPoisson on every rank of a z-slab split, emulated in one process:
    each rank's kernels in turn, the all-to-alls, the global sum and the
    ghost-plane exchange done by copying between the ranks' tensors."""
    import torch
    from pascal_poisson_fft_b200 import dist as D
    dev = torch.device("cuda", 0)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    m = p.metrics
    dmx1, dmx2, dmx3, dx3 = t(m["dmx1"]), t(m["dmx2"]), t(m["dmx3"]), t(m["dx3"])
    slabs = [D.SlabPoisson(p.n1m, p.n2m, p.n3m, p.L1, p.L2, p.pbc, r, nranks, dev) for r in range(nranks)]
    Ps = [torch.zeros(s.ghost_shape(), dtype=torch.float64, device=dev) for s in slabs]
    for s in slabs:
        s.forward(t(p.f[s.z0:s.z0 + s.rows]))
        s.coefficients(dx3, dmx3)
    n_sys = slabs[0].spec.shape[1]
    sends = []
    for s in slabs:
        a_rd, c_rd, d_rd = (torch.empty((2, n_sys), dtype=torch.float64, device=dev) for _ in range(3))
        D._Kernels.modified(s.a, s.b, s.c, s.spec, a_rd, c_rd, d_rd)
        sends.append(D.pack_reduced(a_rd, c_rd, d_rd, nranks))
    backs = []
    for k in range(nranks):
        ra, rb, rc, rd = D.reduced_systems(torch.stack([snd[k] for snd in sends]))
        D._Kernels.solve(ra, rb, rc, rd)
        backs.append(D.pack_solution(rd))
    for k, s in enumerate(slabs):
        D._Kernels.update(s.a, s.c, s.spec, D.unpack_solution(torch.stack([bk[k] for bk in backs]), n_sys))
        s.inverse(Ps[k])
    total = sum(float(s.local_sum(P).item()) for s, P in zip(slabs, Ps))
    shift = torch.tensor([total / (p.n1m * p.n2m * p.n3m)], dtype=torch.float64, device=dev)
    for s, P in zip(slabs, Ps):
        s.shift(P, shift)
    periodic = bool(p.pbc[2])
    for k, (s, P) in enumerate(zip(slabs, Ps)):
        lo = k - 1 if k > 0 else (nranks - 1 if periodic else None)
        hi = k + 1 if k < nranks - 1 else (0 if periodic else None)
        if lo is not None:
            P[0] = Ps[lo][slabs[lo].rows]
        if hi is not None:
            P[s.rows + 1] = Ps[hi][1]
    for s, P in zip(slabs, Ps):
        s.ghosts(P, dmx1, dmx2, dmx3)
    full = torch.zeros((p.n3m + 2, p.n2m + 2, p.n1m + 2), dtype=torch.float64, device=dev)
    full[0] = Ps[0][0]
    for s, P in zip(slabs, Ps):
        full[1 + s.z0:1 + s.z0 + s.rows] = P[1:s.rows + 1]
    full[p.n3m + 1] = Ps[-1][slabs[-1].rows + 1]
    torch.cuda.synchronize()
    return full.cpu().numpy()


@pytest.mark.parametrize("pbc,shape,nranks", [((1, 1, 0), (64, 48, 40), 2), ((0, 0, 0), (48, 32, 33), 4),
                                              ((0, 1, 0), (32, 40, 24), 3), ((1, 0, 0), (40, 32, 64), 8),
                                              ((1, 1, 1), (32, 32, 32), 4)])
def test_slab_solve_matches_single_gpu_and_oracle(pbc, shape, nranks):
    from _util import gpu_solve, oracle_solve, rel_l2
    from pascal_poisson_fft_b200 import workloads as W
    rng = np.random.default_rng(sum(shape) + nranks)
    p = W.random_problem(rng, *shape, pbc, beta=1.5 if not pbc[2] else 0.0)
    full = _emulated_slab_solve(p, nranks)
    # the multi-rank TDMA eliminates in another order than Thomas, so the
    # ill-conditioned low modes agree to cond * eps rather than bit for bit
    assert rel_l2(full, gpu_solve(p)) < 1e-10
    assert rel_l2(full, oracle_solve(p)) < 1e-10
