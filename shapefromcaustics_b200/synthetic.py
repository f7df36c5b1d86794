"""Seeded synthetic photon sets with the workloads' shapes and value distributions.

The reference's photons come from OptiX tracing (``model/caustics.py:242-291``), which is not
part of this library; these generators stand in for it. All draws are float64 from a
``torch.Generator`` in a fixed order, cast to float32 at the end, so a (seed, device) pair
always gives the same photons.

Photon parameterisation (shared by every generator): a photon at pixel position ``p`` with
pixel-space differential ``D = R(theta) diag(s1, s2)`` is passed to the splat as
``xp = 2 p / (W, H) - 1`` (the reference's corner convention, ``photon_differentials.cu:39-44``),
``Mp[:, :2] = D^-1 diag(W/2, H/2)`` and ``Mp[:, 2] = 0`` (the splat support is then the
ellipse with semi-axes s1, s2 pixels), ``radius = 2 max(s1, s2) / W`` (so the reference's box
half-width ``ceil(radius W / 2)`` covers the ellipse) -- the same quantities
``model/caustics.py:224-239`` derives from traced differentials.
"""
import math

import torch

__all__ = ["photons_from_pixels", "uniform_cluster_photons", "caustic_curve_photons",
           "batch_specs", "batch_photons", "upstream_grad"]


def _gen(seed, device):
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    return g


def photons_from_pixels(pos, theta, s1, s2, energy, H, W, channel=None):
    """Splat inputs from pixel-space photon parameters (float64 tensors, any device)."""
    n = pos.shape[1]
    dev = pos.device
    c, s = torch.cos(theta), torch.sin(theta)
    # D^-1 = diag(1/s1, 1/s2) R(-theta)
    M = torch.zeros((2, 3, n), dtype=torch.float64, device=dev)
    M[0, 0] = c / s1 * (W / 2.0)
    M[0, 1] = s / s1 * (H / 2.0)
    M[1, 0] = -s / s2 * (W / 2.0)
    M[1, 1] = c / s2 * (H / 2.0)
    xp = torch.empty((2, n), dtype=torch.float64, device=dev)
    xp[0] = 2.0 * pos[0] / W - 1.0
    xp[1] = 2.0 * pos[1] / H - 1.0
    radius = 2.0 * torch.maximum(s1, s2) / W
    cp = (torch.zeros((1, n), dtype=torch.int64, device=dev) if channel is None
          else channel.reshape(1, n).to(torch.int64))
    return (energy.to(torch.float32).contiguous(), xp.to(torch.float32).contiguous(),
            M.to(torch.float32).contiguous(), cp.contiguous(), radius.to(torch.float32).contiguous())


def _loguniform(g, n, lo, hi, device):
    u = torch.rand(n, generator=g, dtype=torch.float64, device=device)
    return torch.exp(math.log(lo) + u * (math.log(hi) - math.log(lo)))


def uniform_cluster_photons(n=2 ** 20, H=512, W=512, seed=0, s_range=(0.5, 4.0), clusters=8,
                            sigma=20.0, energy=(0.5, 1.0), device="cpu"):
    """Half uniform over the image, half in Gaussian clusters (sigma px) around uniformly
    placed centres; differentials R(theta) diag(s1, s2) with theta ~ U[0, pi) and
    s ~ logU[s_range]; energy ~ U[energy]. Order shuffled."""
    g = _gen(seed, device)
    f64 = dict(dtype=torch.float64, device=device)
    size = torch.tensor([[W], [H]], **f64)
    n_uni = n // 2
    n_cl = n - n_uni
    pos_uni = torch.rand((2, n_uni), generator=g, **f64) * size
    centres = torch.rand((2, clusters), generator=g, **f64) * size
    which = torch.randint(0, clusters, (n_cl,), generator=g, device=device)
    pos_cl = centres[:, which] + torch.randn((2, n_cl), generator=g, **f64) * sigma
    pos = torch.cat([pos_uni, pos_cl], dim=1)
    perm = torch.randperm(n, generator=g, device=device)
    pos = pos[:, perm]
    theta = torch.rand(n, generator=g, **f64) * math.pi
    s1 = _loguniform(g, n, s_range[0], s_range[1], device)
    s2 = _loguniform(g, n, s_range[0], s_range[1], device)
    e = energy[0] + torch.rand(n, generator=g, **f64) * (energy[1] - energy[0])
    return photons_from_pixels(pos, theta, s1, s2, e, H, W)


def caustic_curve_photons(n=2 ** 26, H=2048, W=2048, seed=0, curve_fraction=0.8, curves=4,
                          width_px=1.5, s_range=(0.25, 16.0), energy=(0.5, 1.0), device="cpu"):
    """Contention workload: ``curve_fraction`` of the photons on ``curves`` sinusoidal caustic
    curves with a Gaussian cross-section of ``width_px``, the rest uniform. Each curve spans
    the image width with amplitude ~H/10 and 6-10 periods (about 4 image widths of arc), so
    the curves' +-2 sigma bands cover about 5% of the image."""
    g = _gen(seed, device)
    f64 = dict(dtype=torch.float64, device=device)
    n_curve = int(round(n * curve_fraction))
    n_uni = n - n_curve
    size = torch.tensor([[W], [H]], **f64)
    pos_uni = torch.rand((2, n_uni), generator=g, **f64) * size
    which = torch.randint(0, curves, (n_curve,), generator=g, device=device)
    centre = (torch.arange(curves, **f64) + 0.5) / curves * H
    amp = (0.08 + 0.04 * torch.rand(curves, generator=g, **f64)) * H
    freq = 6.0 + 4.0 * torch.rand(curves, generator=g, **f64)
    phase = torch.rand(curves, generator=g, **f64) * 2 * math.pi
    xs = torch.rand(n_curve, generator=g, **f64) * W
    ys = centre[which] + amp[which] * torch.sin(2 * math.pi * freq[which] * xs / W + phase[which])
    noise = torch.randn((2, n_curve), generator=g, **f64) * width_px
    pos_curve = torch.stack([xs, ys]) + noise
    pos = torch.cat([pos_uni, pos_curve], dim=1)
    perm = torch.randperm(n, generator=g, device=device)
    pos = pos[:, perm]
    theta = torch.rand(n, generator=g, **f64) * math.pi
    s1 = _loguniform(g, n, s_range[0], s_range[1], device)
    s2 = _loguniform(g, n, s_range[0], s_range[1], device)
    e = energy[0] + torch.rand(n, generator=g, **f64) * (energy[1] - energy[0])
    return photons_from_pixels(pos, theta, s1, s2, e, H, W)


def batch_specs(n_sims=64, seed=0, n_range=(2 ** 16, 2 ** 22), sizes=(256, 512, 1024)):
    """Uneven batch: photon counts ~ logU[n_range], square image edges drawn from ``sizes``.
    Returns a list of ``(n_photons, (1, H, W))``."""
    g = _gen(seed, "cpu")
    u = torch.rand(n_sims, generator=g, dtype=torch.float64)
    counts = torch.exp(math.log(n_range[0]) + u * (math.log(n_range[1]) - math.log(n_range[0])))
    pick = torch.randint(0, len(sizes), (n_sims,), generator=g)
    return [(int(round(float(c))), (1, sizes[int(k)], sizes[int(k)])) for c, k in zip(counts, pick)]


def batch_photons(specs, seed=0, device="cpu", **kw):
    """Concatenated photons of a batch (each simulation drawn with its own seed)."""
    parts = [uniform_cluster_photons(n, H, W, seed=seed * 1000003 + s, device=device, **kw)
             for s, (n, (C, H, W)) in enumerate(specs)]
    return tuple(torch.cat([p[k] for p in parts], dim=-1).contiguous() for k in range(5))


def upstream_grad(shape, seed=1, device="cpu"):
    """i.i.d. N(0, 1) upstream gradient image (float32)."""
    g = _gen(seed, device)
    return torch.randn(tuple(shape), generator=g, dtype=torch.float64, device=device).to(torch.float32)
