"""Seeded synthetic problems (the workloads the solver is measured and tested on).

No public dataset is involved: every right-hand side is generated from a
seed with numpy's PCG64 generator, with the shapes, grids and spectra the
benchmark configurations name.  Cell centres are the midpoints of the
reference's faces (01_Fortran/examples/mpi_subdomain.f90:397-472; the
right-hand-side kernel of module_solve_poisson.f90:155-167 uses the same
midpoints).  Every field is returned as a float64 array of shape
(n3m, n2m, n1m) (Fortran f(1:n1m,1:n2m,1:n3m)).

A Neumann-z problem is solvable only if f has zero volume-weighted mean
(sum_k dx3_k * mean_xy f_k = 0); the generators remove that mean so the
answer does not depend on which row the gauge pins.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import mesh

TWO_PI = 2.0 * np.pi


@dataclass
class Problem:
    name: str
    n1m: int
    n2m: int
    n3m: int
    L1: float
    L2: float
    L3: float
    pbc: tuple
    beta: float                      # z stretch (0 = uniform); gamma = 2 beta
    f: np.ndarray | None = None
    metrics: dict = field(default_factory=dict)   # dmx1, dmx2, dmx3, dx3, x1, x2, x3

    @property
    def shape(self):
        return (self.n3m, self.n2m, self.n1m)

    @property
    def cells(self) -> int:
        return self.n1m * self.n2m * self.n3m


def build_metrics(p: Problem) -> Problem:
    x1, _, dmx1 = mesh(p.n1m, p.L1, True, 0.0, p.pbc[0])
    x2, _, dmx2 = mesh(p.n2m, p.L2, True, 0.0, p.pbc[1])
    uni = p.beta == 0.0
    x3, dx3, dmx3 = mesh(p.n3m, p.L3, uni, 2.0 * p.beta, p.pbc[2])
    p.metrics = dict(dmx1=dmx1, dmx2=dmx2, dmx3=dmx3, dx3=dx3, x1=x1, x2=x2, x3=x3)
    return p


def centres(p: Problem):
    m = p.metrics
    xc = 0.5 * (m["x1"][1:p.n1m + 1] + m["x1"][2:p.n1m + 2])
    yc = 0.5 * (m["x2"][1:p.n2m + 1] + m["x2"][2:p.n2m + 2])
    zc = 0.5 * (m["x3"][1:p.n3m + 1] + m["x3"][2:p.n3m + 2])
    return xc, yc, zc


def remove_volume_mean(f: np.ndarray, dx3: np.ndarray) -> np.ndarray:
    n3m = f.shape[0]
    w = dx3[1:n3m + 1]
    plane = f.mean(axis=(1, 2))
    f -= (plane * w).sum() / w.sum()
    return f


def config1(seed: int = 1, n: int = 64) -> Problem:
    """[0,2pi)^2 x [0,1], periodic x,y, Neumann z, uniform;
    f = sin x cos 2y cos(pi z) + N(0, 1e-3)."""
    p = build_metrics(Problem("c1", n, n, n, TWO_PI, TWO_PI, 1.0, (True, True, False), 0.0))
    xc, yc, zc = centres(p)
    rng = np.random.Generator(np.random.PCG64(seed))
    f = np.sin(xc)[None, None, :] * np.cos(2 * yc)[None, :, None] * np.cos(np.pi * zc)[:, None, None]
    f = f + rng.normal(0.0, 1e-3, size=p.shape)
    p.f = remove_volume_mean(f, p.metrics["dx3"])
    return p


def config2(seed: int = 2, n: int = 256, beta: float = 2.0, modes: int = 32) -> Problem:
    """Neumann x,y (DCT) on [0,2pi)^2, tanh z (beta); a seeded sum of Neumann-
    compatible cosines cos(p x/2) cos(q y/2) cos(r pi z) with N(0,1) amplitudes
    plus N(0, 1e-2) noise."""
    p = build_metrics(Problem("c2", n, n, n, TWO_PI, TWO_PI, 1.0, (False, False, False), beta))
    xc, yc, zc = centres(p)
    rng = np.random.Generator(np.random.PCG64(seed))
    A = rng.normal(size=modes)
    pq = rng.integers(0, 17, size=(modes, 2))
    r = rng.integers(0, 9, size=modes)
    f = np.zeros(p.shape)
    for m in range(modes):
        fz = np.cos(r[m] * np.pi * zc)
        fy = np.cos(pq[m, 1] * yc / 2.0)
        fx = np.cos(pq[m, 0] * xc / 2.0)
        f += A[m] * fz[:, None, None] * (fy[:, None] * fx[None, :])[None]
    f += rng.normal(0.0, 1e-2, size=p.shape)
    p.f = remove_volume_mean(f, p.metrics["dx3"])
    return p


def config3(seed: int = 3, n1m: int = 512, n2m: int = 512, n3m: int = 512, beta: float = 1.5,
            modes: int = 48, noise: float = 1e-3, generate=True) -> Problem:
    """Periodic x,y on [0,2pi)^2, tanh z (beta); random Fourier modes with an
    amplitude ~ |k|^-2 spectrum and random phases, plus white noise."""
    p = build_metrics(Problem("c3", n1m, n2m, n3m, TWO_PI, TWO_PI, 1.0, (True, True, False), beta))
    if generate:
        p.f = config3_field(p, seed, modes, noise)
    return p


def config3_field(p: Problem, seed: int, modes: int = 48, noise: float = 1e-3, device=None):
    """The config-3 right-hand side; evaluated with torch on `device` when
    given (fast for 512^3), else with numpy.  Returns a numpy array, or a
    torch tensor when device is given."""
    rng = np.random.Generator(np.random.PCG64(seed))
    kx = rng.integers(0, 17, size=modes)
    ky = rng.integers(-16, 17, size=modes)
    kz = rng.integers(0, 9, size=modes)
    kk = np.sqrt(kx ** 2 + ky ** 2 + (np.pi * kz) ** 2) + 1.0
    amp = rng.normal(size=modes) / kk ** 2
    ph = rng.uniform(0, TWO_PI, size=modes)
    xc, yc, zc = centres(p)
    if device is None:
        f = np.zeros(p.shape)
        for m in range(modes):
            cxv, sxv = np.cos(kx[m] * xc + ph[m]), np.sin(kx[m] * xc + ph[m])
            cyv, syv = np.cos(ky[m] * yc), np.sin(ky[m] * yc)
            plane = cyv[:, None] * cxv[None, :] - syv[:, None] * sxv[None, :]
            f += amp[m] * np.cos(kz[m] * np.pi * zc)[:, None, None] * plane[None]
        f += rng.normal(0.0, noise, size=p.shape)
        return remove_volume_mean(f, p.metrics["dx3"])
    import torch
    t = lambda a: torch.as_tensor(a, dtype=torch.float64, device=device)
    X, Y, Z = t(xc), t(yc), t(zc)
    f = torch.zeros(p.shape, dtype=torch.float64, device=device)
    for m in range(modes):
        plane = torch.cos(ky[m] * Y)[:, None] * torch.cos(kx[m] * X + ph[m])[None, :] \
            - torch.sin(ky[m] * Y)[:, None] * torch.sin(kx[m] * X + ph[m])[None, :]
        f += amp[m] * torch.cos(kz[m] * np.pi * Z)[:, None, None] * plane[None]
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    f += noise * torch.randn(p.shape, dtype=torch.float64, device=device, generator=g)
    w = t(p.metrics["dx3"][1:p.n3m + 1])
    f -= (f.mean(dim=(1, 2)) * w).sum() / w.sum()
    return f


C4_XY = (48, 64, 96, 128, 160, 192, 256, 320, 384)
C4_Z = (32, 64, 128, 256)


def config4(seed: int = 4, count: int = 96, generate: bool = True, device=None):
    """Batched uneven problems: Nx, Ny drawn from C4_XY (radix 2, 3, 5), Nz
    from C4_Z, periodic or Neumann (DCT) per problem in x and y, Neumann z,
    uniform z spacing, on [0,2pi)^2 x [0,1].  Right-hand sides are seeded
    Gaussian fields smoothed by a 3-point (1/4, 1/2, 1/4) filter along each
    axis (wrapping on periodic axes, mirrored at walls), mean removed.
    With `device`, fields are torch tensors made there."""
    rng = np.random.Generator(np.random.PCG64(seed))
    probs = []
    for k in range(count):
        nx, ny = int(rng.choice(C4_XY)), int(rng.choice(C4_XY))
        nz = int(rng.choice(C4_Z))
        pbc = (bool(rng.integers(2)), bool(rng.integers(2)), False)
        probs.append(build_metrics(Problem(f"c4_{k}", nx, ny, nz, TWO_PI, TWO_PI, 1.0, pbc, 0.0)))
    if generate:
        for k, p in enumerate(probs):
            p.f = config4_field(p, seed * 1000 + k, device)
    return probs


def config4_field(p: Problem, seed: int, device=None):
    """The config-4 right-hand side of one problem (numpy, or torch on `device`)."""
    if device is None:
        g = np.random.Generator(np.random.PCG64(seed)).standard_normal(p.shape)
        for ax, per in ((2, p.pbc[0]), (1, p.pbc[1]), (0, p.pbc[2])):
            lo = np.roll(g, 1, axis=ax)
            hi = np.roll(g, -1, axis=ax)
            if not per:   # mirror at the walls: the outside neighbour is the cell itself
                idx = [slice(None)] * 3
                idx[ax] = 0
                lo[tuple(idx)] = g[tuple(idx)]
                idx[ax] = -1
                hi[tuple(idx)] = g[tuple(idx)]
            g = 0.25 * lo + 0.5 * g + 0.25 * hi
        return remove_volume_mean(g, p.metrics["dx3"])
    import torch
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    g = torch.randn(p.shape, dtype=torch.float64, device=device, generator=gen)
    for ax, per in ((2, p.pbc[0]), (1, p.pbc[1]), (0, p.pbc[2])):
        lo = torch.roll(g, 1, dims=ax)
        hi = torch.roll(g, -1, dims=ax)
        if not per:
            lo.select(ax, 0).copy_(g.select(ax, 0))
            hi.select(ax, g.shape[ax] - 1).copy_(g.select(ax, g.shape[ax] - 1))
        g = 0.25 * lo + 0.5 * g + 0.25 * hi
    w = torch.as_tensor(p.metrics["dx3"][1:p.n3m + 1], dtype=torch.float64, device=device)
    g -= (g.mean(dim=(1, 2)) * w).sum() / w.sum()
    return g


def config5(seed: int = 5, n1m: int = 256, n2m: int = 256, n3m: int = 128, beta: float = 2.0,
            modes: int = 48, noise: float = 1e-3):
    """Differentiation workload: periodic x,y, tanh z (beta); the right-hand
    side f and the right-hand side f_tgt whose solve is the target u_tgt of
    J = 1/2 ||u - u_tgt||^2, both seeded random-mode fields (config3_field).
    Returns (problem with f, f_tgt)."""
    p = build_metrics(Problem("c5", n1m, n2m, n3m, TWO_PI, TWO_PI, 1.0, (True, True, False), beta))
    p.f = config3_field(p, seed, modes, noise)
    return p, config3_field(p, seed + 1000, modes, noise)


def manufactured(n: int, pbc=(True, True, False), L: float = 2.0):
    """u = cos(pi x) cos(pi y) cos(pi z) on [0,L]^3 with f = -3 pi^2 u
    (module_solve_poisson.f90:127-209); exact for the continuous problem."""
    p = build_metrics(Problem("mms", n, n, n, L, L, L, tuple(pbc), 0.0))
    xc, yc, zc = centres(p)
    u = np.cos(np.pi * zc)[:, None, None] * np.cos(np.pi * yc)[None, :, None] * np.cos(np.pi * xc)[None, None, :]
    p.f = -3.0 * np.pi ** 2 * u
    return p, u


def random_problem(rng: np.random.Generator, n1m, n2m, n3m, pbc, beta=0.0, L1=TWO_PI, L2=TWO_PI, L3=1.0,
                   compatible=True) -> Problem:
    p = build_metrics(Problem("rand", n1m, n2m, n3m, L1, L2, L3, tuple(pbc), beta))
    f = rng.standard_normal(p.shape)
    p.f = remove_volume_mean(f, p.metrics["dx3"]) if compatible else f
    return p
