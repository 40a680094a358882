"""Parity at the benchmark's own size: the 512^3 config-3 problem (periodic x,y,
Neumann z on a tanh grid with beta = 1.5, random Fourier modes with a |k|^-2
spectrum plus white noise), solved through the C ABI in FP64 and in mixed
precision with one FP64 refinement sweep (the bench's setting), each compared
with the FP64 oracle on the same right-hand side."""
import numpy as np
import pytest

from _util import gpu_solve, oracle_solve, rel_l2
from pascal_poisson_fft_b200 import PPF_MIXED
from pascal_poisson_fft_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL64 = 1e-12      # FP64 path vs the FP64 oracle, rel-L2 over the ghosted field
TOL_MIXED = 1e-10  # mixed + refinement vs the FP64 oracle


@pytest.fixture(scope="module")
def c3_512():
    import torch
    p = W.config3(generate=False)
    p.f = W.config3_field(p, seed=3, device=torch.device("cuda", 0)).cpu().numpy()
    return p, oracle_solve(p)


def test_fp64_512cube_matches_oracle(c3_512):
    p, R = c3_512
    assert rel_l2(gpu_solve(p), R) < TOL64


def test_mixed_one_sweep_512cube_matches_oracle(c3_512):
    p, R = c3_512
    assert rel_l2(gpu_solve(p, precision=PPF_MIXED, max_sweeps=1), R) < TOL_MIXED
