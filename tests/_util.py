"""Helpers shared by the tests: run a Problem through the oracle or libppf."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O


def oracle_solve(p, nthreads=0, imag_zero=True):
    m = p.metrics
    return O.poisson_solve(p.f, p.L1, p.L2, p.pbc, m["dmx1"], m["dmx2"], m["dmx3"], m["dx3"],
                           cpu_fft1_imag_zero=imag_zero, nthreads=nthreads)


def gpu_solve(p, precision=0, max_sweeps=-1, sweep_tol=0.0, plan=None, return_plan=False, lowk_threshold=0.0):
    import torch
    import pascal_poisson_fft_b200 as ppf
    m = p.metrics
    dev = torch.device("cuda", 0)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    if plan is None:
        plan = ppf.Plan(p.n1m, p.n2m, p.n3m, p.L1, p.L2, *p.pbc, precision=precision,
                        max_sweeps=max_sweeps, sweep_tol=sweep_tol, lowk_threshold=lowk_threshold)
    f = t(p.f)
    P = torch.zeros((p.n3m + 2, p.n2m + 2, p.n1m + 2), dtype=torch.float64, device=dev)
    plan.solve(f, P, t(m["dmx1"]), t(m["dmx2"]), t(m["dmx3"]), t(m["dx3"]))
    torch.cuda.synchronize()
    out = P.cpu().numpy()
    return (out, plan) if return_plan else out


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))
