"""torch.autograd.Function over the hand-written adjoint of the shift-and-sum.

``sum_objective(shifts, plan)`` returns J(s) = sum_w h w |sum_k F_k e^{i w.s_k}|^2
for sum shifts ``shifts`` (nframe x 2, float64) of a plan whose spectra are
computed (mc_plan_forward); its backward is the gradient the adjoint kernel
produces in one pass over the spectra (mc_plan_objective).  The forward and
the backward both run in libmc; torch only carries the values.
"""
from __future__ import annotations

import torch


class SumObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, shifts: torch.Tensor, plan) -> torch.Tensor:
        J, grad, _ = plan.objective(shifts.detach().to("cpu", torch.float64).numpy())
        ctx.save_for_backward(torch.from_numpy(grad).to(shifts.device, shifts.dtype))
        return shifts.new_tensor(J)

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        (grad,) = ctx.saved_tensors
        return grad_out * grad, None


def sum_objective(shifts: torch.Tensor, plan) -> torch.Tensor:
    return SumObjective.apply(shifts, plan)
