"""Reference-shaped API, host-array API and error behaviour on the GPU."""
import numpy as np
import pytest

from _util import gpu_solve, oracle_solve, rel_l2
import pascal_poisson_fft_b200 as ppf
from pascal_poisson_fft_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def test_reference_shaped_calls_match_handle_api():
    import torch
    rng = np.random.default_rng(31)
    p = W.random_problem(rng, 32, 24, 20, (1, 0, 0), beta=1.0)
    m = p.metrics
    ppf.fft_poisson_plan_cuda_create(p.n1m + 1, p.n2m + 1, p.n3m + 1, p.L1, p.L2, p.L3, *p.pbc)
    ppf.cuda_Poisson_FFT_initial()
    PRHS = _dev(p.f)
    P = torch.zeros(p.n3m + 2, p.n2m + 2, p.n1m + 2, dtype=torch.float64, device="cuda")
    ppf.cuda_Poisson_FFT_1D(PRHS, P, _dev(m["dmx1"]), _dev(m["dmx2"]), _dev(m["dmx3"]), _dev(m["dx3"]))
    ppf.cuda_Poisson_FFT_clean()
    assert np.array_equal(PRHS.cpu().numpy(), p.f)      # input left intact
    assert np.array_equal(P.cpu().numpy(), gpu_solve(p))


def test_host_array_solve():
    rng = np.random.default_rng(32)
    p = W.random_problem(rng, 48, 32, 40, (0, 1, 0), beta=0.0)
    m = p.metrics
    plan = ppf.Plan(p.n1m, p.n2m, p.n3m, p.L1, p.L2, *p.pbc)
    P = plan.solve_host(p.f, m["dmx1"], m["dmx2"], m["dmx3"], m["dx3"])
    assert rel_l2(P, oracle_solve(p)) < 1e-12


def test_host_array_async_two_plans():
    """ppf_solve_host_async on two plans and two streams, alternating over
    different right-hand sides (page-locked host tensors)."""
    import torch
    rng = np.random.default_rng(34)
    probs = [W.random_problem(rng, 40, 32, 24, (1, 1, 0), beta=1.5) for _ in range(4)]
    p0 = probs[0]
    m = p0.metrics
    plans = [ppf.Plan(p0.n1m, p0.n2m, p0.n3m, p0.L1, p0.L2, *p0.pbc) for _ in range(2)]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    mh = [torch.as_tensor(np.ascontiguousarray(m[k])).pin_memory() for k in ("dmx1", "dmx2", "dmx3", "dx3")]
    fh = [torch.as_tensor(q.f).pin_memory() for q in probs]
    Ph = [torch.empty(p0.gshape if hasattr(p0, "gshape") else (p0.n3m + 2, p0.n2m + 2, p0.n1m + 2),
                      dtype=torch.float64).pin_memory() for _ in probs]
    for i in range(len(probs)):
        plans[i % 2].solve_host_async(fh[i], Ph[i], *mh, stream=streams[i % 2])
    torch.cuda.synchronize()
    for q, P in zip(probs, Ph):
        q.metrics = m
        assert rel_l2(P.numpy(), oracle_solve(q)) < 1e-12


def test_nan_rhs_is_reported():
    rng = np.random.default_rng(33)
    p = W.random_problem(rng, 16, 16, 16, (1, 1, 0))
    p.f[3, 4, 5] = np.nan
    P, plan = gpu_solve(p, return_plan=True)
    with pytest.raises(ppf.PPFError) as e:
        plan.last_sweeps()
    assert e.value.code == -6


def test_wrong_sizes_rejected():
    import torch
    plan = ppf.Plan(16, 16, 16, 1.0, 1.0)
    f = torch.zeros(15, 16, 16, dtype=torch.float64, device="cuda")
    P = torch.zeros(18, 18, 18, dtype=torch.float64, device="cuda")
    m = torch.zeros(18, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        plan.solve(f, P, m, m, m, m)
