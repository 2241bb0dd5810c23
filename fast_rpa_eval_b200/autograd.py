"""torch.autograd wrappers over the C-ABI forward / adjoint pairs.

* ``rho1(P1, plan, wave, gwave, bias, gbias, n_active)`` -> (rho1, grad rho1);
  backward is ``frpa_rho1_adjoint_p1`` (dL/dP1 from both outputs' upstream
  gradients).  phi is re-read in the backward; nothing of the forward is saved.
* ``sumup(Q, plan, lhmfd, mrs, opr, spline, delta_v0, n_active)`` -> delta_v;
  backward is ``frpa_sumup_adjoint_q`` (dL/dQ_lm).

Only P1 and Q carry gradients; every other argument is a constant of the
problem.  All tensors are flat float64 CUDA tensors in the reference layouts.
"""

from __future__ import annotations

import torch

from . import _lib


class _Rho1(torch.autograd.Function):
    @staticmethod
    def forward(ctx, P1, plan, wave, gwave, bias, gbias, n_active):
        T = plan.T
        d = plan.desc
        rho = torch.empty(d.n_full_points * T, dtype=torch.float64, device=P1.device)
        grad = torch.empty(3 * d.n_max_batch_size * d.n_my_batches_work * T, dtype=torch.float64, device=P1.device)
        plan.execute(n_active, wave, gwave, P1.detach(), bias, gbias, rho, grad,
                     stream=torch.cuda.current_stream(P1.device))
        ctx.plan, ctx.wave, ctx.gwave, ctx.n_active, ctx.P1_shape = plan, wave, gwave, n_active, P1.shape
        return rho, grad

    @staticmethod
    def backward(ctx, g_rho, g_grad):
        dP1 = torch.zeros(ctx.P1_shape, dtype=torch.float64, device=ctx.wave.device)
        g_rho = None if g_rho is None else g_rho.contiguous()
        g_grad = None if g_grad is None else g_grad.contiguous()
        if g_rho is not None or g_grad is not None:
            ctx.plan.adjoint_p1(ctx.n_active, ctx.wave, ctx.gwave, g_rho, g_grad, dP1,
                                stream=torch.cuda.current_stream(dP1.device))
        return dP1, None, None, None, None, None, None


class _Sumup(torch.autograd.Function):
    @staticmethod
    def forward(ctx, Q, plan, lhmfd, mrs, opr, spline, delta_v0, n_active):
        dv = delta_v0.detach().clone()
        plan.execute(n_active, lhmfd, mrs, opr, Q.detach(), spline, dv, stream=torch.cuda.current_stream(Q.device))
        ctx.plan, ctx.lhmfd, ctx.mrs, ctx.opr, ctx.n_active = plan, lhmfd, mrs, opr, n_active
        ctx.save_for_backward(Q)
        return dv

    @staticmethod
    def backward(ctx, g):
        (Q,) = ctx.saved_tensors
        dQ = torch.empty_like(Q)
        ctx.plan.adjoint_q(ctx.n_active, ctx.lhmfd, ctx.mrs, ctx.opr, Q.detach(), g.contiguous(), dQ,
                           stream=torch.cuda.current_stream(Q.device))
        return dQ, None, None, None, None, None, None, None


def rho1(P1, plan: _lib.Rho1Plan, wave, gwave, bias, gbias, n_active: int):
    return _Rho1.apply(P1, plan, wave, gwave, bias, gbias, n_active)


def sumup(Q, plan: _lib.SumupPlan, lhmfd, mrs, opr, spline, delta_v0, n_active: int):
    return _Sumup.apply(Q, plan, lhmfd, mrs, opr, spline, delta_v0, n_active)
