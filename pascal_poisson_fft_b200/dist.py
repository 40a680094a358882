"""Tridiagonal systems whose rows are split over ranks (z slabs): the
multi-rank path of PaScaL_TDMA_many_solve_cuda
(01_Fortran/PaScaL_TDMA/src/pascal_tdma_cuda.f90:243-266), one rank per GPU.

Each rank holds rows [r0, r0 + n_row) of every system (arrays of shape
(n_row, n_sys), system index fastest, float64 CUDA tensors):

1. ppf_tdma_many_modified: the modified Thomas sweep reduces every system
   to the rank's first and last rows (2 reduced rows per system, b = 1);
2. all-to-all: each rank receives, for its slice of the systems, the
   reduced rows of all ranks (2 * nranks rows, rank-major), in place of the
   reference's MPI_Alltoall transposes (transpose_slab_xy_to_yz);
3. ppf_tdma_many on the reduced systems;
4. all-to-all back of the reduced solution (transpose_slab_yz_to_xy);
5. ppf_tdma_many_update finishes the local rows.

The exchange uses torch.distributed (NCCL between GPUs).  Everything that
computes runs in libppf's kernels; torch only moves the reduced rows.
"""
from __future__ import annotations

import ctypes

from . import PPFError, _check, _dptr, _stream_ptr, lib


class _Kernels:
    """The per-rank steps, in libppf (CUDA tensors)."""

    @staticmethod
    def modified(a, b, c, d, a_rd, c_rd, d_rd):
        n_row, n_sys = d.shape
        ptrs = [_dptr(t, nm, n_row * n_sys) for t, nm in ((a, "a"), (b, "b"), (c, "c"), (d, "d"))]
        ptrs += [_dptr(t, nm, 2 * n_sys) for t, nm in ((a_rd, "a_rd"), (c_rd, "c_rd"), (d_rd, "d_rd"))]
        _check("ppf_tdma_many_modified", lib().ppf_tdma_many_modified(*ptrs, n_sys, n_row, _stream_ptr(None)))

    @staticmethod
    def solve(a, b, c, d):
        n_row, n_sys = d.shape
        ptrs = [_dptr(t, nm, n_row * n_sys) for t, nm in ((a, "a"), (b, "b"), (c, "c"), (d, "d"))]
        _check("ppf_tdma_many", lib().ppf_tdma_many(*ptrs, n_sys, n_row, _stream_ptr(None)))

    @staticmethod
    def update(a, c, d, x_rd):
        n_row, n_sys = d.shape
        ptrs = [_dptr(t, nm, n_row * n_sys) for t, nm in ((a, "a"), (c, "c"), (d, "d"))]
        ptrs.append(_dptr(x_rd, "x_rd", 2 * n_sys))
        _check("ppf_tdma_many_update", lib().ppf_tdma_many_update(*ptrs, n_sys, n_row, _stream_ptr(None)))


def _host_staged(group) -> bool:
    """Whether collectives of `group` need their CUDA tensors staged through
    host memory (gloo moves host tensors; NCCL moves device memory)."""
    import torch.distributed as dist
    return dist.get_backend(group) == "gloo"


def _torch_exchange(group):
    import torch
    import torch.distributed as dist
    staged = _host_staged(group)

    def exchange(send):
        if staged and send.is_cuda:
            host = send.cpu()
            recv = torch.empty_like(host)
            dist.all_to_all_single(recv, host, group=group)
            return recv.to(send.device)
        recv = torch.empty_like(send)
        dist.all_to_all_single(recv, send, group=group)
        return recv
    return exchange


def all_reduce_sum(t, group=None):
    """In-place sum over the ranks of `group` (through host memory on gloo)."""
    import torch.distributed as dist
    if _host_staged(group) and t.is_cuda:
        h = t.cpu()
        dist.all_reduce(h, group=group)
        t.copy_(h)
    else:
        dist.all_reduce(t, group=group)


def pack_reduced(a_rd, c_rd, d_rd, nranks):
    """Send buffer of the reduced rows: [destination rank, (a, c, d), row, system
    of the destination's slice]; systems are split into nranks contiguous
    slices (zero-padded to equal size: a padded system solves to 0)."""
    import torch
    n_sys = a_rd.shape[1]
    per = -(-n_sys // nranks)
    buf = torch.zeros((3, 2, nranks * per), dtype=a_rd.dtype, device=a_rd.device)
    buf[0, :, :n_sys] = a_rd
    buf[1, :, :n_sys] = c_rd
    buf[2, :, :n_sys] = d_rd
    return buf.view(3, 2, nranks, per).permute(2, 0, 1, 3).contiguous()


def reduced_systems(recv):
    """The reduced systems of this rank's slice from the received buffer
    [source rank, (a, c, d), row, system]: (2 * nranks, per) arrays, rows in
    rank order, b = 1."""
    import torch
    nranks, _, _, per = recv.shape
    a = recv[:, 0].reshape(2 * nranks, per).contiguous()
    c = recv[:, 1].reshape(2 * nranks, per).contiguous()
    d = recv[:, 2].reshape(2 * nranks, per).contiguous()
    b = torch.ones_like(a)
    return a, b, c, d


def pack_solution(x_rt):
    """[destination rank, row, system of this slice] from the (2*nranks, per) solution."""
    two_n, per = x_rt.shape
    return x_rt.view(two_n // 2, 2, per).contiguous()


def unpack_solution(recv, n_sys):
    """The reduced solution (2, n_sys) of this rank's rows from
    [source rank (= system slice), row, system]."""
    nranks, _, per = recv.shape
    return recv.permute(1, 0, 2).reshape(2, nranks * per)[:, :n_sys].contiguous()


def tdma_many_dist(a, b, c, d, group=None, exchange=None, kernels=_Kernels):
    """Solve in place (d <- x) the systems whose rows this rank holds, arrays
    (n_row, n_sys) with n_row >= 3.  Every rank of `group` calls it with the
    same n_sys; a, c are overwritten with the modified coefficients (as the
    reference does).  `exchange(send) -> recv` is the all-to-all of
    equally split first dimensions (torch.distributed by default)."""
    import torch
    import torch.distributed as dist
    n_row, n_sys = d.shape
    if n_row < 3:
        raise PPFError("tdma_many_dist", -1, f"n_row {n_row} < 3 rows on this rank")
    nranks = dist.get_world_size(group) if exchange is None else exchange.nranks
    ex = exchange if exchange is not None else _torch_exchange(group)
    a_rd, c_rd, d_rd = (torch.empty((2, n_sys), dtype=d.dtype, device=d.device) for _ in range(3))
    kernels.modified(a, b, c, d, a_rd, c_rd, d_rd)
    ra, rb, rc, rd = reduced_systems(ex(pack_reduced(a_rd, c_rd, d_rd, nranks)))
    kernels.solve(ra, rb, rc, rd)
    x_rd = unpack_solution(ex(pack_solution(rd)), n_sys)
    kernels.update(a, c, d, x_rd)


def slab_rows(n3m: int, nranks: int, rank: int):
    """(z0, rows) of rank `rank` when n3m z rows are split over nranks (the
    first n3m % nranks ranks take one row more)."""
    base, extra = divmod(n3m, nranks)
    rows = base + (1 if rank < extra else 0)
    z0 = rank * base + min(rank, extra)
    return z0, rows


def halo_ops(rank, nranks, periodic):
    """The point-to-point messages of one ghost-plane exchange, in posting
    order: ("send", plane, peer) / ("recv", plane, peer), planes indexed in
    the ghosted layout (0 and n+1 are the ghost planes, 1 and n the first
    and last interior ones; n is passed symbolically as -1 and n+1 as -2).

    Messages between one pair of ranks are matched in posting order (NCCL
    ignores tags), so the order is chosen to be right even when both
    neighbours are the same rank (two ranks with periodic z): sends go out as
    (first plane -> lower neighbour, last plane -> upper neighbour) and
    receives are posted as (upper ghost <- upper neighbour, lower ghost <-
    lower neighbour).  The k-th plane a rank sends to a peer then lands in
    the k-th plane that peer receives from it: a rank's first plane fills
    the upper ghost of the rank below it, its last plane the lower ghost of
    the rank above it."""
    lo = rank - 1 if rank > 0 else (nranks - 1 if periodic else None)
    hi = rank + 1 if rank < nranks - 1 else (0 if periodic else None)
    ops = []
    if lo is not None:
        ops.append(("send", 1, lo))
    if hi is not None:
        ops.append(("send", -1, hi))
    if hi is not None:
        ops.append(("recv", -2, hi))
    if lo is not None:
        ops.append(("recv", 0, lo))
    return ops


def halo_exchange(P, rank, nranks, periodic, group=None):
    """Ghost planes between slabs: this rank's first and last interior z
    planes to the neighbours' upper and lower ghost planes (whole planes of
    the ghosted layout), wrapping around when z is periodic.  A single
    periodic rank copies its own planes."""
    import torch.distributed as dist
    n = P.shape[0] - 2
    if nranks == 1:
        if periodic:
            P[0].copy_(P[n])
            P[n + 1].copy_(P[1])
        return
    idx = {0: 0, 1: 1, -1: n, -2: n + 1}
    staged = _host_staged(group) and P.is_cuda
    ops, landed = [], []
    for kind, plane, peer in halo_ops(rank, nranks, periodic):
        if kind == "send":
            buf = P[idx[plane]].cpu() if staged else P[idx[plane]].contiguous()
            ops.append(dist.P2POp(dist.isend, buf, peer, group))
        else:
            buf = P[idx[plane]].cpu() if staged else P[idx[plane]]
            ops.append(dist.P2POp(dist.irecv, buf, peer, group))
            landed.append((idx[plane], buf))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    if staged:
        for k, buf in landed:
            P[k].copy_(buf)


class SlabPoisson:
    """One rank's part of the z-slab FP64 Poisson solve (the reference's
    np1 = np2 = 1, np3 = nranks decomposition): x and y transforms on the
    rank's z rows, the multi-rank TDMA along z, the global mean and the
    ghost planes from the neighbours.  f, P (ghosted) and dmx3, dx3 slices
    are this rank's; dmx3_g, dx3_g are the global metric arrays."""

    def __init__(self, n1m, n2m, n3m, L1, L2, pbc, rank, nranks, device=None):
        import torch
        from . import PPF_FP64, Plan
        self.rank, self.nranks = rank, nranks
        self.n = (n1m, n2m, n3m)
        self.pbc = tuple(int(bool(v)) for v in pbc)
        self.z0, self.rows = slab_rows(n3m, nranks, rank)
        if self.rows < 3:
            raise PPFError("SlabPoisson", -1, f"rank {rank} holds {self.rows} z rows; at least 3 are needed")
        self.plan = Plan(n1m, n2m, self.rows, L1, L2, *self.pbc, precision=PPF_FP64)
        ns = ctypes.c_int()
        _check("ppf_slab_systems", lib().ppf_slab_systems(self.plan._h, ctypes.byref(ns)))
        dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        kw = dict(dtype=torch.float64, device=dev)
        self.spec = torch.empty((self.rows, ns.value), **kw)
        self.a, self.b, self.c = (torch.empty((self.rows, ns.value), **kw) for _ in range(3))
        self.sum = torch.zeros(1, **kw)

    def ghost_shape(self):
        n1m, n2m, _ = self.n
        return (self.rows + 2, n2m + 2, n1m + 2)

    # ---- rank-local steps (libppf kernels) ----
    def forward(self, f):
        _check("ppf_slab_forward", lib().ppf_slab_forward(self.plan._h, _dptr(f, "f"), self.spec.data_ptr(),
                                                          _stream_ptr(None)))

    def coefficients(self, dx3_g, dmx3_g):
        _check("ppf_slab_coefficients", lib().ppf_slab_coefficients(
            self.plan._h, self.a.data_ptr(), self.b.data_ptr(), self.c.data_ptr(), self.spec.data_ptr(),
            _dptr(dx3_g, "dx3_g", self.n[2] + 2), _dptr(dmx3_g, "dmx3_g", self.n[2] + 2), self.z0, self.n[2],
            _stream_ptr(None)))

    def inverse(self, P):
        _check("ppf_slab_inverse", lib().ppf_slab_inverse(self.plan._h, self.spec.data_ptr(), _dptr(P, "P"),
                                                          _stream_ptr(None)))

    def local_sum(self, P):
        _check("ppf_slab_sum", lib().ppf_slab_sum(self.plan._h, _dptr(P, "P"), self.sum.data_ptr(),
                                                  _stream_ptr(None)))
        return self.sum

    def shift(self, P, shift):
        _check("ppf_slab_shift", lib().ppf_slab_shift(self.plan._h, _dptr(P, "P"), _dptr(shift, "shift", 1),
                                                      _stream_ptr(None)))

    def ghosts(self, P, dmx1, dmx2, dmx3_g):
        dmx3 = dmx3_g[self.z0:self.z0 + self.rows + 2].contiguous()
        _check("ppf_slab_ghosts", lib().ppf_slab_ghosts(
            self.plan._h, _dptr(P, "P"), _dptr(dmx1, "dmx1"), _dptr(dmx2, "dmx2"), _dptr(dmx3, "dmx3"),
            int(self.rank == 0), int(self.rank == self.nranks - 1), _stream_ptr(None)))

    # ---- the whole solve over torch.distributed ----
    def solve(self, f, P, dmx1, dmx2, dmx3_g, dx3_g, group=None):
        """The whole slab solve, collective over `group` (NCCL between GPUs;
        on a gloo group the exchanges are staged through host memory)."""
        self.forward(f)
        self.coefficients(dx3_g, dmx3_g)
        tdma_many_dist(self.a, self.b, self.c, self.spec, group=group)
        self.inverse(P)
        s = self.local_sum(P).clone()
        all_reduce_sum(s, group)
        s /= float(self.n[0] * self.n[1] * self.n[2])
        self.shift(P, s)
        halo_exchange(P, self.rank, self.nranks, bool(self.pbc[2]), group)
        self.ghosts(P, dmx1, dmx2, dmx3_g)
