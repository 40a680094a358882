"""FP64 parity of the CUDA solve (through the C ABI) against the oracle."""
import os

import numpy as np
import pytest

from _util import gpu_solve, oracle_solve, rel_l2
from oracle import oracle as O
from pascal_poisson_fft_b200 import workloads as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL64 = 1e-12   # FP64 path vs the FP64 oracle, rel-L2 over the ghosted field


def test_golden_fixture_cases():
    import pascal_poisson_fft_b200 as ppf
    g = np.load(os.path.join(GOLD, "solve_npref.npz"))
    for i in range(int(g["ncases"])):
        n1, n2, n3, p1, p2, p3 = (int(v) for v in g[f"{i}_meta"])
        L1, L2, L3 = g[f"{i}_L"]
        p = W.Problem("gold", n1, n2, n3, L1, L2, L3, (bool(p1), bool(p2), bool(p3)), 0.0)
        p.f = g[f"{i}_f"]
        p.metrics = {k: g[f"{i}_{k}"] for k in ("dmx1", "dmx2", "dmx3", "dx3")}
        P = gpu_solve(p)
        assert rel_l2(P, g[f"{i}_P"]) < TOL64, (i, (n1, n2, n3), (p1, p2, p3))


@pytest.mark.parametrize("shape", [(768, 16, 6), (16, 768, 6), (1024, 8, 4), (8, 1024, 4), (640, 20, 5)])
@pytest.mark.parametrize("pbc", [(1, 1, 0), (0, 0, 0)])
def test_fp64_long_lines(shape, pbc):
    """Longest transform lines (tiles of 48 KB and more of shared memory)."""
    rng = np.random.default_rng(hash((shape, pbc)) & 0xffff)
    p = W.random_problem(rng, *shape, pbc, beta=1.0)
    assert rel_l2(gpu_solve(p), oracle_solve(p)) < TOL64


@pytest.mark.parametrize("shape", [(16, 12, 10), (32, 32, 32), (48, 40, 24), (96, 80, 33), (40, 30, 100),
                                   (20, 24, 513)])
@pytest.mark.parametrize("pbc", [(1, 1, 0), (0, 0, 0), (0, 1, 0), (1, 0, 0), (1, 1, 1)])
@pytest.mark.parametrize("beta", [0.0, 2.0])
def test_fp64_matches_oracle(shape, pbc, beta):
    if pbc[2] and beta:
        pytest.skip("stretching applies to wall-bounded z")
    rng = np.random.default_rng(hash((shape, pbc, beta)) & 0xffff)
    p = W.random_problem(rng, *shape, pbc, beta=beta)
    P = gpu_solve(p)
    R = oracle_solve(p)
    assert rel_l2(P, R) < TOL64


def test_config1_64cube():
    p = W.config1()
    P = gpu_solve(p)
    R = oracle_solve(p)
    assert rel_l2(P, R) < TOL64


def test_config2_256cube_dct_stretched():
    p = W.config2()
    P = gpu_solve(p)
    R = oracle_solve(p)
    assert rel_l2(P, R) < TOL64


def test_eigenvector_kat():
    n = 64
    p = W.config1(n=n)
    xc, yc, zc = W.centres(p)
    p.f = np.sin(xc)[None, None, :] * np.cos(2 * yc)[None, :, None] * np.cos(np.pi * zc)[:, None, None]
    h, dz = 2 * np.pi / n, 1.0 / n
    lam = 2 * (1 - np.cos(h)) / h ** 2 + 2 * (1 - np.cos(2 * h)) / h ** 2 + 4 * np.sin(np.pi / (2 * n)) ** 2 / dz ** 2
    P = gpu_solve(p)
    np.testing.assert_allclose(P[1:-1, 1:-1, 1:-1], -p.f / lam, rtol=0, atol=1e-14)


def test_manufactured_second_order():
    errs = []
    for n in (16, 32, 64, 128):
        p, u = W.manufactured(n)
        P = gpu_solve(p)
        errs.append(np.sqrt(np.mean((P[1:-1, 1:-1, 1:-1] - u) ** 2)))
    rates = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert np.all(rates > 1.9), (errs, rates)


def test_residual_and_mean_at_large_size():
    """Size-independent properties at 256^2 x 128: zero arithmetic mean and an
    FP64-level residual of the operator the solve inverts."""
    rng = np.random.default_rng(123)
    p = W.random_problem(rng, 256, 256, 128, (1, 1, 0), beta=2.0)
    P = gpu_solve(p)
    m = p.metrics
    r = O.residual(p.f, P, p.L1, p.L2, p.pbc, m["dmx3"], m["dx3"])
    assert np.linalg.norm(r) / np.linalg.norm(p.f) < 1e-11
    assert abs(P[1:-1, 1:-1, 1:-1].mean()) < 1e-13


def test_linearity():
    rng = np.random.default_rng(4)
    p = W.random_problem(rng, 64, 48, 40, (0, 1, 0), beta=1.0)
    q = W.random_problem(rng, 64, 48, 40, (0, 1, 0), beta=1.0)
    a, b = 0.75, -2.5
    Pp = gpu_solve(p)
    Pq = gpu_solve(q)
    p.f = a * p.f + b * q.f
    Ps = gpu_solve(p)
    assert rel_l2(Ps, a * Pp + b * Pq) < 1e-13


def test_repeat_is_deterministic():
    rng = np.random.default_rng(8)
    p = W.random_problem(rng, 64, 64, 64, (1, 1, 0), beta=1.5)
    P1, plan = gpu_solve(p, return_plan=True)
    P2 = gpu_solve(p, plan=plan)
    assert np.array_equal(P1, P2)


@pytest.mark.parametrize("nz", [32, 47, 64, 97, 200, 256, 300, 512])
@pytest.mark.parametrize("pbc", [(1, 1, 0), (0, 0, 0), (0, 1, 0)])
def test_fp64_z_lengths(nz, pbc):
    """z lengths that split into uneven row segments in the shared-memory
    partitioned z solve (and its limits), stretched z."""
    rng = np.random.default_rng(nz * 7 + sum(pbc))
    p = W.random_problem(rng, 24, 20, nz, pbc, beta=2.0)
    assert rel_l2(gpu_solve(p), oracle_solve(p)) < TOL64
