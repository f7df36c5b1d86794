"""Autograd face of the splatting op: ``PDS``, with the reference's signature.

Mirror of ``model/photon_differential.py:7-19``: ``PDS.apply(Ep, xp, Mp, cp, radius,
output_size, max_pixel_radius)`` returns the ``[C,H,W]`` photon map and its backward returns
``(grad_Ep, grad_xp, grad_Mp, None, None, None, None)``.

Difference from the reference: the forward's photon binning and sort (the plan) is kept for
the backward instead of being recomputed. ``set_keep_plan(False)`` drops it after the forward
and rebuilds it in the backward, trading one binning pass for the plan's workspace (about 76
bytes per photon) held between the passes.
"""
import torch

from .splatting import SplatPlan

_keep_plan = True


def set_keep_plan(keep: bool):
    global _keep_plan
    _keep_plan = bool(keep)


class PDS(torch.autograd.Function):
    @staticmethod
    def forward(ctx, Ep, xp, Mp, cp, radius, output_size, max_pixel_radius):
        plan = SplatPlan(Ep, xp, Mp, cp, radius, output_size, max_pixel_radius)
        out = plan.forward()
        ctx.save_for_backward(Ep, xp, Mp, cp, radius)
        ctx.output_size = tuple(int(v) for v in output_size)
        ctx.max_pixel_radius = int(max_pixel_radius)
        ctx.plan_ws = plan.ws if _keep_plan else None
        ctx.cfg = plan.cfg
        return out

    @staticmethod
    def backward(ctx, grad_pds):
        Ep, xp, Mp, cp, radius = ctx.saved_tensors
        if ctx.plan_ws is not None:
            plan = SplatPlan.__new__(SplatPlan)
            plan.n = Ep.size(0)
            plan.C, plan.H, plan.W = ctx.output_size
            plan.mpr = ctx.max_pixel_radius
            plan.cfg = ctx.cfg
            plan.device = Ep.device
            plan.inputs = (Ep, xp, Mp, cp, radius)
            plan.ws = ctx.plan_ws
        else:
            plan = SplatPlan(Ep, xp, Mp, cp, radius, ctx.output_size, ctx.max_pixel_radius,
                             config=ctx.cfg)
        grad_Ep, grad_xp, grad_Mp = plan.backward(grad_pds.contiguous())
        ctx.plan_ws = None
        return grad_Ep, grad_xp, grad_Mp, None, None, None, None
