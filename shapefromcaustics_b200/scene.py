"""Scene description of the height-field glass plate and the synthetic height fields of the
workloads.

``PlateScene`` holds the plate's geometry and the light (the quantities ``pds_plate`` carries
to the refraction kernels, ``plate.plate_params``); ``height_field_bumps`` draws the seeded
height fields of the Landweber workloads (a base thickness plus Gaussian bumps);
``fused_silica`` is the glass's dispersion (refractive index per wavelength). Units:
millimetres, wavelengths in micrometres.
"""
import torch

__all__ = ["PlateScene", "height_field_bumps", "fused_silica"]


class PlateScene:
    """Glass plate over a receiver.

    ``texel``: height-field texel size (mm), the field spans ``[-W texel/2, W texel/2]`` in x
    (columns) and the same in y (rows); ``ior``: refractive index; ``receiver_distance``:
    from the flat bottom face (z = 0) to the receiver (mm); ``receiver_half``: half-extent of
    the square receiver (mm); ``light_dir``: unit propagation direction (default straight
    down).
    """

    def __init__(self, texel=0.1, ior=1.5, receiver_distance=50.0, receiver_half=14.08,
                 light_dir=(0.0, 0.0, -1.0)):
        self.texel = float(texel)
        self.ior = float(ior)
        self.receiver_distance = float(receiver_distance)
        self.receiver_half = float(receiver_half)
        d = torch.tensor(light_dir, dtype=torch.float64)
        self.light_dir = tuple((d / d.norm()).tolist())


def height_field_bumps(H, W, seed=0, bumps=32, base=1.0, amp=(0.0, 0.05), width=(4.0, 24.0),
                       dtype=torch.float64, device="cpu"):
    """Base thickness plus Gaussian bumps (amplitude and width uniform in the given ranges,
    width in texels, centres uniform); millimetres."""
    g = torch.Generator(device="cpu").manual_seed(int(seed))
    cy = torch.rand(bumps, generator=g, dtype=torch.float64) * H
    cx = torch.rand(bumps, generator=g, dtype=torch.float64) * W
    a = amp[0] + torch.rand(bumps, generator=g, dtype=torch.float64) * (amp[1] - amp[0])
    w = width[0] + torch.rand(bumps, generator=g, dtype=torch.float64) * (width[1] - width[0])
    yy, xx = torch.meshgrid(torch.arange(H, dtype=torch.float64), torch.arange(W, dtype=torch.float64),
                            indexing="ij")
    h = torch.full((H, W), base, dtype=torch.float64)
    for k in range(bumps):
        h += a[k] * torch.exp(-((yy - cy[k]) ** 2 + (xx - cx[k]) ** 2) / (2 * w[k] ** 2))
    return h.to(dtype=dtype, device=device)


def fused_silica(wavelength_um):
    """Refractive index of fused silica at a wavelength in micrometres: the three-term Sellmeier
    fit the reference uses (``model/caustics.py:13-23``, fitted on 0.21-6.7 um),
    ``n^2 = 1 + sum_k B_k / (1 - (C_k / lambda)^2)`` with B = (0.6961663, 0.4079426,
    0.8974794) and C = (0.0684043, 0.1162414, 9.896161) um. Scalars or tensors."""
    lam = wavelength_um
    terms = ((0.6961663, 0.0684043), (0.4079426, 0.1162414), (0.8974794, 9.896161))
    n2 = 1.0
    for b, c in terms:
        n2 = n2 + b / (1.0 - (c / lam) ** 2)
    return n2 ** 0.5
