"""ppf_tdma_many / ppf_tdma_cycl_many against the reference's tdmas.cpp
(golden fixture) and the oracle restatement of tdmas.f90."""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _gpu(a, b, c, d, cyclic):
    import torch
    import pascal_poisson_fft_b200 as ppf
    t = [torch.as_tensor(np.ascontiguousarray(v), dtype=torch.float64, device="cuda") for v in (a, b, c, d)]
    (ppf.tdma_cycl_many if cyclic else ppf.tdma_many)(*t)
    torch.cuda.synchronize()
    for v, tv in zip((a, b, c), t[:3]):
        assert np.array_equal(v, tv.cpu().numpy())  # coefficients untouched
    return t[3].cpu().numpy()


def test_against_reference_fixture():
    g = np.load(os.path.join(GOLD, "tdma_ref.npz"))
    for i in range(int(g["ncases"])):
        a, b, c, d, x = (g[f"{i}_{k}"] for k in "abcdx")
        got = _gpu(a, b, c, d, str(g[f"{i}_kind"]) == "cycl")
        np.testing.assert_allclose(got, x, rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("n_sys,n_row", [(1, 1), (3, 2), (37, 3), (128, 16), (100, 17), (1000, 64), (513, 255),
                                         (64, 1000), (7, 1024)])
@pytest.mark.parametrize("cyclic", [False, True])
def test_against_oracle(n_sys, n_row, cyclic):
    if cyclic and n_row < 3:
        pytest.skip("cyclic systems need 3 rows")
    rng = np.random.default_rng(n_sys * 7919 + n_row)
    a = rng.uniform(-1, 1, (n_row, n_sys)); c = rng.uniform(-1, 1, (n_row, n_sys))
    b = (np.abs(a) + np.abs(c) + rng.uniform(0.2, 2, (n_row, n_sys))) * rng.choice([-1.0, 1.0], (n_row, n_sys))
    d = rng.standard_normal((n_row, n_sys))
    got = _gpu(a, b, c, d, cyclic)
    ref = [v.copy() for v in (a, b, c, d)]
    O.tdma_many(*ref, cyclic=cyclic)
    assert np.linalg.norm(got - ref[3]) / np.linalg.norm(ref[3]) < 1e-13
