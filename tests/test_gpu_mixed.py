"""Mixed precision (FP32 transforms + FP64 residual refinement) and FP32."""
import numpy as np
import pytest

from _util import gpu_solve, oracle_solve, rel_l2
from pascal_poisson_fft_b200 import PPF_FP32, PPF_MIXED
from pascal_poisson_fft_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL_MIXED = 1e-10   # mixed + refinement vs FP64, rel-L2
TOL_FP32 = 5e-5     # a single FP32 solve vs FP64, rel-L2


@pytest.mark.parametrize("pbc", [(1, 1, 0), (0, 0, 0), (0, 1, 0), (1, 0, 0)])
def test_mixed_matches_oracle(pbc):
    rng = np.random.default_rng(21)
    p = W.random_problem(rng, 64, 48, 64, pbc, beta=1.5)
    R = oracle_solve(p)
    P = gpu_solve(p, precision=PPF_MIXED, max_sweeps=3)
    assert rel_l2(P, R) < TOL_MIXED


@pytest.mark.parametrize("pbc", [(1, 1, 0), (0, 0, 0)])
def test_fp32_single_solve_accuracy(pbc):
    rng = np.random.default_rng(22)
    p = W.random_problem(rng, 64, 64, 64, pbc, beta=1.5)
    R = oracle_solve(p)
    P = gpu_solve(p, precision=PPF_FP32)
    assert rel_l2(P, R) < TOL_FP32


def test_mixed_config3_shape_256():
    p = W.config3(n1m=256, n2m=256, n3m=256)
    P64 = gpu_solve(p)
    P = gpu_solve(p, precision=PPF_MIXED, max_sweeps=2)
    assert rel_l2(P, P64) < TOL_MIXED


def test_sweep_gate_stops_early():
    rng = np.random.default_rng(23)
    p = W.random_problem(rng, 64, 64, 64, (1, 1, 0), beta=1.5)
    P, plan = gpu_solve(p, precision=PPF_MIXED, max_sweeps=6, sweep_tol=1e-9, return_plan=True)
    sweeps, rel = plan.last_sweeps()
    assert 1 <= sweeps < 6 and rel < 1e-9
    R = oracle_solve(p)
    assert rel_l2(P, R) < TOL_MIXED


def test_mixed_mean_is_fp64_zero():
    """The residual cannot see constants; the gauge (zero arithmetic mean) is
    kept in FP64 by the accumulate pass."""
    p = W.config3(n1m=128, n2m=128, n3m=64)
    P = gpu_solve(p, precision=PPF_MIXED, max_sweeps=2)
    u = P[1:-1, 1:-1, 1:-1]
    assert abs(u.mean()) < 1e-14 * np.abs(u).max()


def test_mixed_deterministic():
    rng = np.random.default_rng(24)
    p = W.random_problem(rng, 64, 64, 32, (0, 1, 0), beta=1.0)
    P1, plan = gpu_solve(p, precision=PPF_MIXED, max_sweeps=2, return_plan=True)
    P2 = gpu_solve(p, plan=plan)
    assert np.array_equal(P1, P2)


def test_fp32_768x768x384_radix3():
    """The FP32 single-solve throughput configuration (768x768x384, radix
    3*2^k): the mixed path within 1e-10 of the FP64 solve, and a single FP32
    solve within 2e-4 (its error grows with the grid: ~7e-5 here)."""
    p = W.config3(n1m=768, n2m=768, n3m=384, generate=False)
    import torch
    p.f = W.config3_field(p, 3, device=torch.device("cuda", 0)).cpu().numpy()
    P64 = gpu_solve(p)
    assert rel_l2(gpu_solve(p, precision=PPF_MIXED, max_sweeps=3), P64) < TOL_MIXED
    assert rel_l2(gpu_solve(p, precision=PPF_FP32), P64) < 2e-4


# The FP64 systems of the mixed path (lam * dz_min^2 < lowk_threshold) run in
# their own latency-bound kernel over a compacted list.  A threshold above
# every eigenvalue sends all systems there: several 32-system groups per
# persistent block, real (DCT x and y) and complex storage, columns shorter
# than its prefetch ring and lengths that are no multiple of its chunk.
@pytest.mark.parametrize("shape,pbc,lowk", [
    ((128, 96, 40), (1, 1, 0), 1e12),
    ((48, 40, 37), (0, 0, 0), 1e12),
    ((64, 32, 21), (0, 1, 0), 1e12),
    ((32, 48, 200), (1, 0, 0), 1e-3),
])
def test_mixed_lowk_systems(shape, pbc, lowk):
    rng = np.random.default_rng(21)
    p = W.random_problem(rng, *shape, pbc, beta=1.5)
    ref = oracle_solve(p)
    P = gpu_solve(p, precision=PPF_MIXED, max_sweeps=3, lowk_threshold=lowk)
    assert rel_l2(P, ref) < TOL_MIXED
    assert rel_l2(gpu_solve(p, precision=PPF_FP32, lowk_threshold=lowk), ref) < TOL_FP32


# A refining mixed solve keeps its first iterate (FP32 values) in an FP32
# ghosted field instead of P: the first sweep's residual and accumulate read
# it from there.  Every boundary pair, compile-time and run-time x lengths,
# no sweep (the iterate goes straight to P), one and two sweeps.
@pytest.mark.parametrize("shape,pbc", [
    ((64, 48, 40), (1, 1, 0)),
    ((64, 48, 40), (0, 0, 0)),
    ((40, 36, 24), (1, 0, 0)),
    ((48, 40, 37), (0, 1, 0)),
    ((512, 512, 24), (1, 1, 0)),
    ((512, 256, 16), (0, 1, 0)),
])
def test_mixed_fp32_first_iterate(shape, pbc):
    import pascal_poisson_fft_b200 as ppf
    rng = np.random.default_rng(5)
    p = W.random_problem(rng, *shape, pbc, beta=1.5)
    ref = oracle_solve(p)
    e0 = rel_l2(gpu_solve(p, precision=PPF_MIXED, max_sweeps=0), ref)
    e1 = rel_l2(gpu_solve(p, precision=PPF_MIXED, max_sweeps=1), ref)
    e2 = rel_l2(gpu_solve(p, precision=PPF_MIXED, max_sweeps=2), ref)
    assert e0 < TOL_FP32
    assert e1 < 1e-8 and e1 < e0 * 1e-3
    assert e2 < TOL_MIXED
    n1, n2, n3 = shape
    mk = lambda s: ppf.Plan(n1, n2, n3, p.L1, p.L2, *pbc, precision=PPF_MIXED, max_sweeps=s)
    a, b = mk(0), mk(1)
    assert b.workspace_bytes() - a.workspace_bytes() == 4 * (n1 + 2) * (n2 + 2) * (n3 + 2)
    a.close()
    b.close()


@pytest.mark.parametrize("nz", [32, 47, 97, 300, 512])
@pytest.mark.parametrize("pbc", [(1, 1, 0), (0, 0, 0)])
def test_mixed_z_lengths(nz, pbc):
    rng = np.random.default_rng(nz * 5 + sum(pbc))
    p = W.random_problem(rng, 32, 24, nz, pbc, beta=1.5)
    assert rel_l2(gpu_solve(p, precision=PPF_MIXED, max_sweeps=3), oracle_solve(p)) < TOL_MIXED
