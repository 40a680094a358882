"""The streamed FP32 z solve (k_thomas_stream: TMA ring, twisted sweep per
column, chunk checkpoints in shared memory), at sizes where a standalone
plan uses it -- at least one block of 256 FP32 values of a z row per SM
(148 blocks) -- and in the shapes it has to handle: complex columns (real
and imaginary parts of periodic-x spectra), real columns (DCT x and y), an
odd number of 16-row chunks with a partial last one, and a single chunk.

Each case runs the single FP32 solve, whose error is the streamed bulk's
own (a refinement sweep would absorb a wrong bulk), and the mixed solve
with refinement, both against the oracle."""
import numpy as np
import pytest

from _util import gpu_solve, oracle_solve, rel_l2
from pascal_poisson_fft_b200 import PPF_FP32, PPF_MIXED
from pascal_poisson_fft_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL_MIXED = 1e-10
TOL_FP32 = 5e-5

# (n1m, n2m, n3m, pbc, beta): z rows of ~74k-147k FP32 values (288-576 blocks)
CASES = [
    (256, 256, 200, (1, 1, 0), 1.5),   # complex; 13 chunks (6 lower, 7 upper), the last 8 rows
    (512, 256, 64, (0, 0, 0), 0.0),    # real columns (DCT x and y); 4 chunks
    (384, 256, 97, (1, 0, 0), 2.0),    # complex, DCT y; 7 chunks, the last one row
    (256, 512, 16, (1, 1, 0), 0.0),    # one chunk: the upper half alone
]


@pytest.mark.parametrize("n1m,n2m,n3m,pbc,beta", CASES)
def test_streamed_bulk_fp32(n1m, n2m, n3m, pbc, beta):
    rng = np.random.default_rng(n3m)
    p = W.random_problem(rng, n1m, n2m, n3m, pbc, beta=beta)
    R = oracle_solve(p)
    assert rel_l2(gpu_solve(p, precision=PPF_FP32), R) < TOL_FP32


@pytest.mark.parametrize("n1m,n2m,n3m,pbc,beta", CASES)
def test_streamed_bulk_mixed(n1m, n2m, n3m, pbc, beta):
    rng = np.random.default_rng(n3m + 1)
    p = W.random_problem(rng, n1m, n2m, n3m, pbc, beta=beta)
    R = oracle_solve(p)
    assert rel_l2(gpu_solve(p, precision=PPF_MIXED, max_sweeps=3), R) < TOL_MIXED
