"""torch.autograd binding of the solve and its transpose (a gradient-check
harness over the C ABI: forward = ppf_solve, backward = ppf_solve_adjoint).

    u = PoissonSolve.apply(f, dx3, dmx3, plan, dmx1, dmx2)

returns the interior solution (n3m, n2m, n1m); gradients flow to f, dx3 and
dmx3.  Every computation runs in libppf's kernels.
"""
from __future__ import annotations

import torch

from . import Plan


class PoissonSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, f, dx3, dmx3, plan: Plan, dmx1, dmx2):
        P = torch.empty(plan.gshape, dtype=torch.float64, device=f.device)
        plan.solve(f.contiguous(), P, dmx1, dmx2, dmx3.contiguous(), dx3.contiguous())
        ctx.plan = plan
        ctx.save_for_backward(P, dx3, dmx3, dmx1, dmx2)
        return P[1:-1, 1:-1, 1:-1].contiguous()

    @staticmethod
    def backward(ctx, gu):
        P, dx3, dmx3, dmx1, dmx2 = ctx.saved_tensors
        plan: Plan = ctx.plan
        df = torch.empty(plan.shape, dtype=torch.float64, device=gu.device)
        ddx3 = torch.empty_like(dx3)
        ddmx3 = torch.empty_like(dmx3)
        plan.solve_adjoint(gu.contiguous(), df, dmx1, dmx2, dmx3.contiguous(), dx3.contiguous(), u=P,
                           ddx3=ddx3, ddmx3=ddmx3)
        return df, ddx3, ddmx3, None, None, None
