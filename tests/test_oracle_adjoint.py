"""The oracle's transpose solve and z-metric gradient (CPU): the adjoint
identity <M f, g> = <f, M^T g> against the oracle's own forward solve, and
central finite differences of <g, u(dx3, dmx3)>."""
import numpy as np
import pytest

from oracle import oracle as O
from pascal_poisson_fft_b200 import workloads as W

PBCS = [(1, 1, 0), (0, 0, 0), (0, 1, 0), (1, 0, 0), (1, 1, 1)]


def _args(p):
    m = p.metrics
    return (p.L1, p.L2, p.pbc, m["dmx1"], m["dmx2"], m["dmx3"], m["dx3"])


@pytest.mark.parametrize("pbc", PBCS)
def test_adjoint_identity(pbc):
    rng = np.random.default_rng(101)
    p = W.random_problem(rng, 12, 10, 9, pbc, beta=2.0)
    f = rng.standard_normal(p.shape)
    g = rng.standard_normal(p.shape)
    Mf = O.poisson_solve(f, *_args(p))[1:-1, 1:-1, 1:-1]
    df = O.poisson_adjoint(g, *_args(p))
    lhs, rhs = float((Mf * g).sum()), float((f * df).sum())
    assert abs(lhs - rhs) <= 1e-13 * abs(lhs)


@pytest.mark.parametrize("pbc", PBCS)
def test_metric_gradient_finite_differences(pbc):
    rng = np.random.default_rng(102)
    p = W.random_problem(rng, 12, 10, 9, pbc, beta=2.0)
    m = p.metrics
    f = rng.standard_normal(p.shape)
    g = rng.standard_normal(p.shape)
    u = O.poisson_solve(f, *_args(p))
    _, ddx3, ddmx3 = O.poisson_adjoint(g, *_args(p), u=u)

    def J(dx3, dmx3):
        P = O.poisson_solve(f, p.L1, p.L2, pbc, m["dmx1"], m["dmx2"], dmx3, dx3)
        return float((P[1:-1, 1:-1, 1:-1] * g).sum())

    h = 1e-6
    for grad, which in ((ddx3, "dx3"), (ddmx3, "dmx3")):
        e = rng.standard_normal(grad.shape)
        plus = dict(dx3=m["dx3"], dmx3=m["dmx3"])
        minus = dict(plus)
        plus[which] = plus[which] + h * e
        minus[which] = minus[which] - h * e
        fd = (J(**plus) - J(**minus)) / (2 * h)
        an = float((grad * e).sum())
        assert abs(fd - an) <= 1e-6 * abs(fd), (which, fd, an)


def test_loss_gradient_in_f():
    """J = 1/2 ||u - u_tgt||^2: dJ/df = M^T (u - u_tgt), checked by central differences."""
    rng = np.random.default_rng(103)
    p = W.random_problem(rng, 16, 12, 10, (1, 1, 0), beta=2.0)
    tgt = O.poisson_solve(W.random_problem(rng, 16, 12, 10, (1, 1, 0), beta=2.0).f, *_args(p))[1:-1, 1:-1, 1:-1]
    J = lambda f: 0.5 * float(((O.poisson_solve(f, *_args(p))[1:-1, 1:-1, 1:-1] - tgt) ** 2).sum())
    u = O.poisson_solve(p.f, *_args(p))[1:-1, 1:-1, 1:-1]
    grad = O.poisson_adjoint(u - tgt, *_args(p))
    for _ in range(4):
        e = rng.standard_normal(p.shape)
        fd = (J(p.f + 1e-6 * e) - J(p.f - 1e-6 * e)) / 2e-6
        assert abs(fd - float((grad * e).sum())) <= 1e-6 * abs(fd)
