"""Scene description of the height-field glass plate and the synthetic height fields of the
workloads.

``PlateScene`` holds the plate's geometry and the light (the quantities ``pds_plate`` carries
to the refraction kernels, ``plate.plate_params``); ``height_field_bumps`` draws the seeded
height fields of the Landweber workloads (a base thickness plus Gaussian bumps). Units:
millimetres.
"""
import torch

__all__ = ["PlateScene", "height_field_bumps"]


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
