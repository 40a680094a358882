"""The oracle pinned: against the reference's own compiled Thomas solvers,
against an independent scipy restatement, and against known answers."""
import os

import numpy as np
import pytest

import npref
from oracle import oracle as O
from pascal_poisson_fft_b200 import workloads as W

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 8, 12, 15, 16, 24, 30, 48, 60, 64, 96, 97, 128, 160,
                               192, 256, 320, 384, 512, 768])
def test_fft_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    np.testing.assert_allclose(O.fft_c2c(x, -1), np.fft.fft(x), rtol=0, atol=1e-13 * np.abs(x).sum())
    np.testing.assert_allclose(O.fft_c2c(x, +1), np.fft.ifft(x) * n, rtol=0, atol=1e-13 * np.abs(x).sum())


def test_tdma_matches_reference_binary_fixture():
    """tests/golden/tdma_ref.npz holds outputs of the reference's tdmas.cpp."""
    g = np.load(os.path.join(GOLD, "tdma_ref.npz"))
    for i in range(int(g["ncases"])):
        a, b, c, d, x = (g[f"{i}_{k}"].copy() for k in "abcdx")
        O.tdma_many(a, b, c, d, cyclic=str(g[f"{i}_kind"]) == "cycl")
        np.testing.assert_allclose(d, x, rtol=1e-14, atol=1e-14)


def test_tdma_matches_live_reference():
    ref = O.ref_tdmas()
    if ref is None:
        pytest.skip("reference tdmas.cpp not built (reference tree absent)")
    import ctypes
    dp = ctypes.POINTER(ctypes.c_double)
    rng = np.random.default_rng(3)
    for ns, nr, cyc in [(11, 40, False), (64, 64, True), (1, 1000, False)]:
        a = rng.uniform(-1, 1, (nr, ns)); c = rng.uniform(-1, 1, (nr, ns))
        b = np.abs(a) + np.abs(c) + 1.0
        d = rng.standard_normal((nr, ns))
        arrs = [v.copy() for v in (a, b, c, d)]
        O.tdma_many(*arrs, cyclic=cyc)
        r = [np.ascontiguousarray(v.copy()) for v in (a, b, c, d)]
        (ref.tdma_cycl_many if cyc else ref.tdma_many)(*[v.ctypes.data_as(dp) for v in r], ns, nr)
        assert np.array_equal(arrs[3], r[3])  # same operations, same order: bit-exact


@pytest.mark.parametrize("pbc", [False, True])
@pytest.mark.parametrize("uniform", [True, False])
def test_mesh_matches_restatements(pbc, uniform):
    import pascal_poisson_fft_b200 as ppf
    a = O.mesh(20, 1.0, uniform, 3.0, pbc)
    b = npref.mesh(20, 1.0, uniform, 3.0, pbc)
    c = ppf.mesh(20, 1.0, uniform, 3.0, pbc)
    for u, v, w in zip(a, b, c):
        np.testing.assert_allclose(u, v, rtol=0, atol=1e-15)
        np.testing.assert_allclose(u, w, rtol=0, atol=1e-15)


def test_solve_matches_independent_fixture():
    g = np.load(os.path.join(GOLD, "solve_npref.npz"))
    for i in range(int(g["ncases"])):
        n1, n2, n3, p1, p2, p3 = (int(v) for v in g[f"{i}_meta"])
        L1, L2, _ = g[f"{i}_L"]
        P = O.poisson_solve(g[f"{i}_f"], L1, L2, (p1, p2, p3), g[f"{i}_dmx1"], g[f"{i}_dmx2"],
                            g[f"{i}_dmx3"], g[f"{i}_dx3"], cpu_fft1_imag_zero=True)
        ref = g[f"{i}_P"]
        assert np.linalg.norm(P - ref) / np.linalg.norm(ref) < 1e-13, (i, (n1, n2, n3), (p1, p2, p3))


@pytest.mark.parametrize("pbc", [(1, 1, 0), (0, 0, 0), (0, 1, 0), (1, 0, 0)])
def test_solve_matches_npref_stretched(pbc):
    rng = np.random.default_rng(11)
    p = W.random_problem(rng, 30, 20, 24, pbc, beta=2.0)
    m = p.metrics
    P1 = O.poisson_solve(p.f, p.L1, p.L2, pbc, m["dmx1"], m["dmx2"], m["dmx3"], m["dx3"])
    P2 = npref.solve(p.f, p.L1, p.L2, pbc, m["dmx1"], m["dmx2"], m["dmx3"], m["dx3"])
    assert np.linalg.norm(P1 - P2) / np.linalg.norm(P2) < 1e-13


def test_eigenvector_kat_config1_shape():
    """sin x cos 2y cos(pi z) is an exact eigenvector of the discrete operator
    on the uniform grid: u = -f / (lx(1) + ly(2) + lz(1))."""
    n = 32
    p = W.config1(n=n)
    xc, yc, zc = W.centres(p)
    f = np.sin(xc)[None, None, :] * np.cos(2 * yc)[None, :, None] * np.cos(np.pi * zc)[:, None, None]
    h, dz = 2 * np.pi / n, 1.0 / n
    lam = 2 * (1 - np.cos(h)) / h ** 2 + 2 * (1 - np.cos(2 * h)) / h ** 2 + 4 * np.sin(np.pi / (2 * n)) ** 2 / dz ** 2
    m = p.metrics
    P = O.poisson_solve(f, p.L1, p.L2, p.pbc, m["dmx1"], m["dmx2"], m["dmx3"], m["dx3"])
    np.testing.assert_allclose(P[1:-1, 1:-1, 1:-1], -f / lam, rtol=0, atol=1e-14)


def test_manufactured_second_order():
    errs = []
    for n in (16, 32, 64):
        p, u = W.manufactured(n)
        m = p.metrics
        P = O.poisson_solve(p.f, p.L1, p.L2, p.pbc, m["dmx1"], m["dmx2"], m["dmx3"], m["dx3"])
        errs.append(np.sqrt(np.mean((P[1:-1, 1:-1, 1:-1] - u) ** 2)))
    rates = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert np.all(rates > 1.9), (errs, rates)


@pytest.mark.parametrize("pbc", [(1, 1, 0), (0, 0, 0), (0, 1, 0), (1, 0, 0)])
def test_residual_vanishes_for_compatible_rhs(pbc):
    rng = np.random.default_rng(5)
    p = W.random_problem(rng, 16, 12, 20, pbc, beta=1.5, compatible=True)
    m = p.metrics
    P = O.poisson_solve(p.f, p.L1, p.L2, pbc, m["dmx1"], m["dmx2"], m["dmx3"], m["dx3"])
    r = O.residual(p.f, P, p.L1, p.L2, pbc, m["dmx3"], m["dx3"])
    assert np.linalg.norm(r) / np.linalg.norm(p.f) < 1e-12
    assert abs(P[1:-1, 1:-1, 1:-1].mean()) < 1e-14


def test_ghost_fill_order_matches_npref():
    rng = np.random.default_rng(9)
    for pbc in [(1, 1, 0), (0, 0, 0), (0, 1, 1), (1, 0, 0), (1, 1, 1)]:
        P = rng.standard_normal((7, 6, 9))
        _, _, d1 = npref.mesh(7, 1.0, True, 0, pbc[0])
        _, _, d2 = npref.mesh(4, 1.0, True, 0, pbc[1])
        _, _, d3 = npref.mesh(5, 1.0, False, 3.0, pbc[2])
        A = P.copy(); B = P.copy()
        O.fill_ghosts(A, pbc, d1, d2, d3)
        npref.fill_ghosts(B, pbc, d1, d2, d3)
        assert np.array_equal(A, B)
