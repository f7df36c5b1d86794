"""The reference's projected Landweber update in PyTorch ops. TEST INFRASTRUCTURE ONLY: the
tests hold the fused device update (``pds_landweber_update_f32``) to it; the product never
imports it.

``ext_shrink`` restates ``shape_from_caustics.py:184-189`` (extShrink), ``vcons_heur``
``:228-241`` (VconsHeur) and ``landweber_update_reference`` the update of ``:386-398``.
"""
import math

import torch
import torch.nn.functional as F

__all__ = ["ext_shrink", "vcons_heur", "landweber_update_reference"]


def ext_shrink(x, alpha, a, b):
    """``shape_from_caustics.py:184-189``."""
    zeros = torch.zeros_like(x)
    ones = torch.ones_like(x)
    return torch.max(torch.min(torch.max(torch.abs(x) - alpha, zeros) * torch.sign(x), b * ones),
                     a * ones)


def vcons_heur(x, d1, d2, mask, gamma, radius):
    """``shape_from_caustics.py:228-241``."""
    vx = torch.sum(x)
    xmean = F.avg_pool2d(x[None, None], 2 * radius + 1, stride=1, padding=radius)[0, 0]
    if vx <= d1:
        x = x + mask * xmean * torch.sin(vx / d1 * math.pi) * gamma
    elif vx >= d2:
        x = x - mask * xmean * torch.sin((vx / d2 - 1) * math.pi) * gamma
    return x


def landweber_update_reference(d, grad, mask, params):
    """The reference's update ops (``shape_from_caustics.py:386-398``), out of place."""
    x = d - params.tau * grad
    x = mask * ext_shrink(x, params.tau * params.alpha, params.lower, params.upper)
    return vcons_heur(x, params.d1, params.d2, mask, params.gamma, params.radius)
