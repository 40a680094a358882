"""Batched uneven problems in one graph launch (ppf_batch_*): each problem
against the oracle (FP64) or its own FP64 plan (mixed), graph replay and
re-capture on new pointers, autotuned schedules, and the 96-problem
batched workload."""
import numpy as np
import pytest

from _util import gpu_solve, oracle_solve, rel_l2
from pascal_poisson_fft_b200 import PPF_FP64, PPF_MIXED
from pascal_poisson_fft_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL64 = 1e-12
TOL_MIXED = 1e-10


def _dev():
    import torch
    return torch.device("cuda", 0)


def _t(a):
    import torch
    if isinstance(a, torch.Tensor):
        return a.to(_dev())
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=_dev())


def _run_batch(probs, precision=PPF_FP64, autotune=True, branches=0, max_sweeps=3, batch=None, Ps=None,
               persistent=False):
    import torch
    import pascal_poisson_fft_b200 as ppf
    if batch is None:
        batch = ppf.Batch([dict(n1m=p.n1m, n2m=p.n2m, n3m=p.n3m, L1=p.L1, L2=p.L2, pbc=p.pbc,
                                precision=precision, max_sweeps=max_sweeps) for p in probs],
                          autotune=autotune, branches=branches, persistent=persistent)
    fs = [_t(p.f) for p in probs]
    if Ps is None:
        Ps = [torch.zeros((p.n3m + 2, p.n2m + 2, p.n1m + 2), dtype=torch.float64, device=_dev()) for p in probs]
    ms = [[_t(p.metrics[k]) for p in probs] for k in ("dmx1", "dmx2", "dmx3", "dx3")]
    batch.solve(fs, Ps, *ms)
    torch.cuda.synchronize()
    return batch, Ps


def _small_uneven(seed, count):
    rng = np.random.default_rng(seed)
    sizes = (24, 40, 48, 64, 80, 96)
    probs = []
    for _ in range(count):
        pbc = (int(rng.integers(2)), int(rng.integers(2)), 0)
        probs.append(W.random_problem(rng, int(rng.choice(sizes)), int(rng.choice(sizes)),
                                      int(rng.choice((9, 16, 33))), pbc, beta=float(rng.choice((0.0, 1.5)))))
    return probs


def test_batch_fp64_matches_oracle():
    probs = _small_uneven(301, 10)
    _, Ps = _run_batch(probs)
    for p, P in zip(probs, Ps):
        assert rel_l2(P.cpu().numpy(), oracle_solve(p)) < TOL64, (p.shape, p.pbc)


def test_batch_mixed_matches_fp64_plans():
    probs = _small_uneven(302, 12)
    _, Ps = _run_batch(probs, precision=PPF_MIXED)
    for p, P in zip(probs, Ps):
        assert rel_l2(P.cpu().numpy(), gpu_solve(p)) < TOL_MIXED, (p.shape, p.pbc)


def test_replay_and_recapture():
    import torch
    probs = _small_uneven(303, 6)
    batch, Ps = _run_batch(probs, branches=3)
    first = [P.clone() for P in Ps]
    _run_batch(probs, batch=batch, Ps=Ps)            # replay of the captured graph
    for a, b in zip(first, Ps):
        assert torch.equal(a, b)
    _, Ps2 = _run_batch(probs, batch=batch)          # new output pointers: re-captured
    for a, b in zip(first, Ps2):
        assert torch.equal(a, b)
    info = [batch.info(k) for k in range(len(probs))]
    assert {i["branch"] for i in info} == {0, 1, 2}
    assert all(i["branches"] == 3 for i in info)


def test_autotune_choices_keep_results():
    probs = _small_uneven(304, 8)
    b1, P1 = _run_batch(probs, autotune=True)
    _, P0 = _run_batch(probs, autotune=False)
    for a, b in zip(P1, P0):
        assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-13
    assert all(b1.info(k)["x_order"] in (0, 1, 2) for k in range(len(probs)))


def test_rejects_bad_descriptor():
    import pascal_poisson_fft_b200 as ppf
    with pytest.raises(ppf.PPFError, match="problem 1"):
        ppf.Batch([dict(n1m=32, n2m=32, n3m=16, L1=1.0, L2=1.0), dict(n1m=33, n2m=32, n3m=16, L1=1.0, L2=1.0)])


def test_config4_batch():
    """96 problems, Nx,Ny in {48..384}, Nz in {32..256}, mixed BCs, FP32 + FP64
    refinement: every problem within 1e-10 of its own FP64 plan solve."""
    import torch
    import pascal_poisson_fft_b200 as ppf
    probs = W.config4(device=_dev())
    batch, Ps = _run_batch(probs, precision=PPF_MIXED, max_sweeps=3)
    worst = 0.0
    for p, P in zip(probs, Ps):
        plan = ppf.Plan(p.n1m, p.n2m, p.n3m, p.L1, p.L2, *p.pbc)
        R = torch.empty_like(P)
        plan.solve(p.f, R, *[_t(p.metrics[k]) for k in ("dmx1", "dmx2", "dmx3", "dx3")])
        torch.cuda.synchronize()
        worst = max(worst, float(torch.linalg.norm(P - R) / torch.linalg.norm(R)))
        plan.close()
    assert worst < TOL_MIXED, worst


# ---- the persistent work-queue form (one kernel for the whole batch) ----

def test_persistent_fp64_matches_oracle():
    probs = _small_uneven(311, 10)
    batch, Ps = _run_batch(probs, persistent=True)
    for p, P in zip(probs, Ps):
        assert rel_l2(P.cpu().numpy(), oracle_solve(p)) < TOL64, (p.shape, p.pbc)
    assert all(batch.info(k)["branches"] == 0 and batch.info(k)["x_runtime"] == 1 for k in range(len(probs)))


def test_persistent_mixed_matches_fp64_plans():
    probs = _small_uneven(312, 12)
    _, Ps = _run_batch(probs, precision=PPF_MIXED, persistent=True)
    for p, P in zip(probs, Ps):
        assert rel_l2(P.cpu().numpy(), gpu_solve(p)) < TOL_MIXED, (p.shape, p.pbc)


def test_persistent_periodic_z_and_fp32():
    import pascal_poisson_fft_b200 as ppf
    rng = np.random.default_rng(313)
    probs = [W.random_problem(rng, 32, 24, 16, (1, 1, 1)), W.random_problem(rng, 40, 48, 20, (0, 1, 1)),
             W.random_problem(rng, 64, 32, 33, (1, 0, 0), beta=1.5)]
    _, Ps = _run_batch(probs, persistent=True)
    for p, P in zip(probs, Ps):
        assert rel_l2(P.cpu().numpy(), oracle_solve(p)) < TOL64, (p.shape, p.pbc)
    _, Ps = _run_batch(probs, precision=ppf.PPF_FP32, persistent=True)
    for p, P in zip(probs, Ps):
        assert rel_l2(P.cpu().numpy(), oracle_solve(p)) < 5e-5, (p.shape, p.pbc)


def test_persistent_replay_and_new_pointers():
    import torch
    probs = _small_uneven(314, 6)
    batch, Ps = _run_batch(probs, precision=PPF_MIXED, persistent=True)
    first = [P.clone() for P in Ps]
    _run_batch(probs, batch=batch, Ps=Ps)            # replay
    for a, b in zip(first, Ps):
        assert torch.equal(a, b)
    _, Ps2 = _run_batch(probs, batch=batch)          # new output pointers
    for a, b in zip(first, Ps2):
        assert torch.equal(a, b)


def test_persistent_config4_against_graph():
    """The 96-problem workload in one persistent launch, FP64 and mixed, each
    problem within the tolerance of the graph form's result."""
    import torch
    probs = W.config4(device=_dev())
    for prec, tol in ((PPF_FP64, TOL64), (PPF_MIXED, TOL_MIXED)):
        _, Pg = _run_batch(probs, precision=prec, max_sweeps=2)
        _, Pp = _run_batch(probs, precision=prec, max_sweeps=2, persistent=True)
        worst = max(float(torch.linalg.norm(a - b) / torch.linalg.norm(b)) for a, b in zip(Pp, Pg))
        assert worst < tol, (prec, worst)
