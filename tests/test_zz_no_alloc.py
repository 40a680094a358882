"""The allocation-free solve (ppf_solve_noalloc) against the regular entry point.

Some callers cannot allocate device memory when they solve: a flow solver
that reserved its whole device budget at start-up, or an application whose
device memory belongs to another framework.  ppf_solve_noalloc serves them
from one static device array.  These tests call it through the C ABI on a
sequence of grids -- first, second, first, first -- so the table upload,
the cached-table path (same grid again) and the return to an earlier grid
after another one are all exercised.  ppf_solve_noalloc runs the same
kernels on the same inputs as ppf_plan_create + ppf_solve, so every result
must equal the plan solve's bit for bit, and the FP64 oracle within the
FP64 tolerance.  This file is collected last so a failure here never hides
the other tests.
"""
import ctypes

import numpy as np
import pytest

import pascal_poisson_fft_b200 as ppf
from pascal_poisson_fft_b200 import workloads as W
from _util import gpu_solve, oracle_solve, rel_l2

pytestmark = pytest.mark.gpu
TOL64 = 1e-12   # the FP64 tolerance of the other parity tests


def _noalloc(p):
    import torch
    m = p.metrics
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    d = ppf._Desc(p.n1m, p.n2m, p.n3m, p.L1, p.L2, int(p.pbc[0]), int(p.pbc[1]), int(p.pbc[2]),
                  ppf.PPF_FP64, 0, 0.0, 0.0)
    f = t(p.f)
    P = torch.full((p.n3m + 2, p.n2m + 2, p.n1m + 2), np.nan, dtype=torch.float64, device="cuda")
    args = [x.data_ptr() for x in (f, P, t(m["dmx1"]), t(m["dmx2"]), t(m["dmx3"]), t(m["dx3"]))]
    rc = ppf.lib().ppf_solve_noalloc(ctypes.byref(d), *args, torch.cuda.current_stream().cuda_stream)
    assert rc == 0, ppf.lib().ppf_last_error()
    torch.cuda.synchronize()
    return P.cpu().numpy()


def test_noalloc_equals_plan_solve_over_a_call_sequence():
    rng = np.random.default_rng(77)
    first = W.random_problem(rng, 64, 48, 40, (1, 1, 0), beta=1.5)
    second = W.random_problem(rng, 96, 80, 33, (0, 1, 0), beta=0.0)
    refs = {id(p): (gpu_solve(p), oracle_solve(p)) for p in (first, second)}
    for step, p in enumerate((first, second, first, first)):
        got = _noalloc(p)
        plan_out, oracle_out = refs[id(p)]
        assert np.array_equal(got, plan_out), f"call {step}: differs from the plan solve"
        assert rel_l2(got, oracle_out) < TOL64, f"call {step}: rel-L2 vs oracle"


def test_noalloc_rejects_grids_beyond_its_array():
    d = ppf._Desc(512, 512, 512, 1.0, 1.0, 1, 1, 0, ppf.PPF_FP64, 0, 0.0, 0.0)
    rc = ppf.lib().ppf_solve_noalloc(ctypes.byref(d), 1, 1, 1, 1, 1, 1, None)
    assert rc == -4  # PPF_ERR_UNSUPPORTED, before any device work
    assert b"bytes of work memory" in ppf.lib().ppf_last_error()
