"""The splat's direct caller: photon differentials on the receiver -> splat inputs -> image.

Mirror of ``model/caustics.py:224-239`` (``change_of_basis_matrix``, ``splat_photons``) on
plain ``[3, N]`` tensors:

    Mp     = 2 / (Du . (Dv x n)) * [Dv x n ; n x Du]        (2 x 3 x N)
    radius = 0.5 * max(|Du|, |Dv|)
    Ep     = 4 * flux / |Du x Dv|

so that ``Mp @ Du = (2, 0)`` and ``Mp @ Dv = (0, 2)``: the splat support is the ellipse
``{(a Du + b Dv) / 2 : a^2 + b^2 < 1}``. The reference drops degenerate photons
(``Du . (Dv x n) == 0``) by boolean-mask compaction, which synchronises with the host; here
they keep their slot with channel -1, which the splat kernels skip (zero contribution, zero
gradient), so shapes stay static and nothing waits on the device.
"""
import torch

from .photon_differential import PDS

__all__ = ["change_of_basis_matrix", "splat_inputs", "splat_photons"]


def change_of_basis_matrix(Du, Dv, normal):
    """-> (Mp [2,3,N], good [N] bool). Degenerate photons get a finite placeholder."""
    tmp = torch.cross(Dv, normal, dim=0)
    den = (Du * tmp).sum(0)
    good = den != 0
    factor = 2.0 / torch.where(good, den, torch.ones_like(den))
    Mp = factor * torch.stack((tmp, torch.cross(normal, Du, dim=0)), dim=0)
    return Mp, good


def splat_inputs(Du, Dv, normal, flux, channel):
    """Splat inputs ``(Ep, Mp, cp, radius)`` for photons with receiver-plane differentials.

    ``Du, Dv, normal``: ``[3, N]``; ``flux``: ``[N]``; ``channel``: ``[N]`` int64.
    """
    Mp, good = change_of_basis_matrix(Du, Dv, normal)
    radius = 0.5 * torch.maximum(Du.norm(dim=0), Dv.norm(dim=0))
    area = torch.cross(Du, Dv, dim=0).norm(dim=0)
    Ep = flux / torch.where(good, area, torch.ones_like(area)) * 4
    cp = torch.where(good, channel, torch.full_like(channel, -1)).reshape(1, -1)
    return Ep.contiguous(), Mp.contiguous(), cp.contiguous(), radius.contiguous()


def splat_photons(Du, Dv, normal, flux, positions_xy, channel, output_size, max_pixel_radius=20):
    """``model/caustics.py:233-239``: splat photons given their receiver-plane position
    ``positions_xy [2, N]`` (normalised receiver coordinates) and differentials."""
    Ep, Mp, cp, radius = splat_inputs(Du, Dv, normal, flux, channel)
    return PDS.apply(Ep, positions_xy.contiguous(), Mp, cp, radius, tuple(output_size),
                     max_pixel_radius)
