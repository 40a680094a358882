"""Transpose solve and z-metric gradient on the GPU (ppf_solve_adjoint):
against the oracle's transpose, the adjoint identity with the oracle's
forward solve, the mixed path against FP64, and the differentiation
workload (256x256x128, tanh z beta=2) against central finite differences."""
import numpy as np
import pytest

from _util import rel_l2
from oracle import oracle as O
from pascal_poisson_fft_b200 import PPF_FP64, PPF_MIXED
from pascal_poisson_fft_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL64 = 1e-12      # FP64 transpose vs the oracle's, rel-L2
TOL_METRIC = 1e-10  # FP64 metric gradient vs the oracle's, rel-L2
TOL_FD = 1e-6      # gradients vs central finite differences (h = 1e-6), relative


def _dev():
    import torch
    return torch.device("cuda", 0)


def _t(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=_dev())


def _args(p):
    m = p.metrics
    return (p.L1, p.L2, p.pbc, m["dmx1"], m["dmx2"], m["dmx3"], m["dx3"])


def _gpu_adjoint(p, g, u=None, precision=PPF_FP64, plan=None):
    import torch
    import pascal_poisson_fft_b200 as ppf
    m = p.metrics
    if plan is None:
        plan = ppf.Plan(p.n1m, p.n2m, p.n3m, p.L1, p.L2, *p.pbc, precision=precision, max_sweeps=3)
    df = torch.empty(p.shape, dtype=torch.float64, device=_dev())
    ddx3 = torch.empty(p.n3m + 2, dtype=torch.float64, device=_dev())
    ddmx3 = torch.empty(p.n3m + 2, dtype=torch.float64, device=_dev())
    if u is None:
        plan.solve_adjoint(_t(g), df, _t(m["dmx1"]), _t(m["dmx2"]), _t(m["dmx3"]), _t(m["dx3"]))
        torch.cuda.synchronize()
        return df.cpu().numpy()
    plan.solve_adjoint(_t(g), df, _t(m["dmx1"]), _t(m["dmx2"]), _t(m["dmx3"]), _t(m["dx3"]), u=_t(u),
                       ddx3=ddx3, ddmx3=ddmx3)
    torch.cuda.synchronize()
    return df.cpu().numpy(), ddx3.cpu().numpy(), ddmx3.cpu().numpy()


@pytest.mark.parametrize("pbc,shape", [((1, 1, 0), (32, 24, 20)), ((0, 0, 0), (32, 24, 20)),
                                       ((0, 1, 0), (40, 30, 33)), ((1, 0, 0), (24, 40, 17)),
                                       ((1, 1, 1), (32, 32, 24))])
def test_adjoint_matches_oracle(pbc, shape):
    rng = np.random.default_rng(201)
    p = W.random_problem(rng, *shape, pbc, beta=2.0)
    g = rng.standard_normal(p.shape)
    u = O.poisson_solve(p.f, *_args(p))
    R, rx, rm = O.poisson_adjoint(g, *_args(p), u=u)
    df, dx, dm = _gpu_adjoint(p, g, u=u)
    assert rel_l2(df, R) < TOL64
    assert rel_l2(dx, rx) < TOL_METRIC
    assert rel_l2(dm, rm) < TOL_METRIC


def test_adjoint_identity_with_oracle_forward():
    rng = np.random.default_rng(202)
    p = W.random_problem(rng, 48, 40, 36, (1, 1, 0), beta=1.5)
    f = rng.standard_normal(p.shape)
    g = rng.standard_normal(p.shape)
    Mf = O.poisson_solve(f, *_args(p))[1:-1, 1:-1, 1:-1]
    df = _gpu_adjoint(p, g)
    lhs, rhs = float((Mf * g).sum()), float((f * df).sum())
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_adjoint_in_place():
    import torch
    import pascal_poisson_fft_b200 as ppf
    rng = np.random.default_rng(203)
    p = W.random_problem(rng, 32, 32, 16, (1, 1, 0), beta=1.0)
    m = p.metrics
    g = rng.standard_normal(p.shape)
    plan = ppf.Plan(p.n1m, p.n2m, p.n3m, p.L1, p.L2, *p.pbc)
    a = _t(g)
    plan.solve_adjoint(a, a, _t(m["dmx1"]), _t(m["dmx2"]), _t(m["dmx3"]), _t(m["dx3"]))
    torch.cuda.synchronize()
    assert rel_l2(a.cpu().numpy(), O.poisson_adjoint(g, *_args(p))) < TOL64


def test_mixed_adjoint_matches_fp64():
    rng = np.random.default_rng(204)
    p = W.random_problem(rng, 64, 64, 48, (1, 1, 0), beta=2.0)
    g = rng.standard_normal(p.shape)
    u = O.poisson_solve(p.f, *_args(p))
    d64, x64, m64 = _gpu_adjoint(p, g, u=u)
    dmx, xmx, mmx = _gpu_adjoint(p, g, u=u, precision=PPF_MIXED)
    assert rel_l2(dmx, d64) < 1e-10
    assert rel_l2(xmx, x64) < 1e-8
    assert rel_l2(mmx, m64) < 1e-8


def test_rejects_metric_gradient_without_u():
    import torch
    import pascal_poisson_fft_b200 as ppf
    p = W.random_problem(np.random.default_rng(205), 16, 16, 8, (1, 1, 0))
    m = p.metrics
    plan = ppf.Plan(p.n1m, p.n2m, p.n3m, p.L1, p.L2, *p.pbc)
    df = torch.empty(p.shape, dtype=torch.float64, device=_dev())
    gx = torch.empty(p.n3m + 2, dtype=torch.float64, device=_dev())
    with pytest.raises(ppf.PPFError):
        plan.solve_adjoint(_t(p.f), df, _t(m["dmx1"]), _t(m["dmx2"]), _t(m["dmx3"]), _t(m["dx3"]), ddx3=gx)


@pytest.mark.parametrize("precision", [PPF_FP64, PPF_MIXED])
def test_config5_finite_differences(precision):
    """256x256x128, periodic x,y, tanh z beta=2: J = 1/2 ||u - u_tgt||^2 through
    the autograd harness; dJ/df and dJ/d dx3 against central differences of
    FP64 solves (h = 1e-6) along 64 random directions each."""
    import torch
    import pascal_poisson_fft_b200 as ppf
    from pascal_poisson_fft_b200.autograd import PoissonSolve
    p, f_tgt = W.config5()
    m = p.metrics
    dev = _dev()
    plan64 = ppf.Plan(p.n1m, p.n2m, p.n3m, p.L1, p.L2, *p.pbc)
    plan = plan64 if precision == PPF_FP64 else ppf.Plan(p.n1m, p.n2m, p.n3m, p.L1, p.L2, *p.pbc,
                                                         precision=precision, max_sweeps=3)
    dmx1, dmx2 = _t(m["dmx1"]), _t(m["dmx2"])
    dmx3, dx3 = _t(m["dmx3"]), _t(m["dx3"])
    Pt = torch.empty(plan64.gshape, dtype=torch.float64, device=dev)
    plan64.solve(_t(f_tgt), Pt, dmx1, dmx2, dmx3, dx3)
    u_tgt = Pt[1:-1, 1:-1, 1:-1].clone()

    f = _t(p.f).requires_grad_(True)
    x3 = dx3.clone().requires_grad_(True)
    u = PoissonSolve.apply(f, x3, dmx3, plan, dmx1, dmx2)
    J = 0.5 * ((u - u_tgt) ** 2).sum()
    J.backward()
    gf, gx = f.grad.detach(), x3.grad.detach()

    P = torch.empty(plan64.gshape, dtype=torch.float64, device=dev)

    def Jeval(ff, xx):
        plan64.solve(ff, P, dmx1, dmx2, dmx3, xx)
        return 0.5 * float(((P[1:-1, 1:-1, 1:-1] - u_tgt) ** 2).sum())

    gen = torch.Generator(device=dev)
    gen.manual_seed(55)
    h = 1e-6
    f0 = f.detach()
    worst_f = worst_x = 0.0
    for _ in range(64):
        e = torch.randn(p.shape, dtype=torch.float64, device=dev, generator=gen)
        fd = (Jeval(f0 + h * e, dx3) - Jeval(f0 - h * e, dx3)) / (2 * h)
        worst_f = max(worst_f, abs(fd - float((gf * e).sum())) / abs(fd))
        ex = torch.randn(p.n3m + 2, dtype=torch.float64, device=dev, generator=gen)
        ex[0] = 0.0
        ex[-1] = 0.0
        fd = (Jeval(f0, dx3 + h * ex) - Jeval(f0, dx3 - h * ex)) / (2 * h)
        worst_x = max(worst_x, abs(fd - float((gx * ex).sum())) / abs(fd))
    assert worst_f < TOL_FD, worst_f
    assert worst_x < TOL_FD, worst_x
