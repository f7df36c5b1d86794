"""Refraction-to-receiver step in float64 on the CPU: its height-field gradient (autograd
through the refraction chain, the FP64 oracle's splat backward at the end) against central
finite differences of the FP64 forward."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import refraction_chain as RF


class OraclePDS(torch.autograd.Function):
    """The splat with the FP64 oracle in both directions (test-only)."""

    @staticmethod
    def forward(ctx, Ep, xp, Mp, cp, radius, shape, mpr):
        ctx.save_for_backward(Ep, xp, Mp, cp, radius)
        ctx.mpr = mpr
        a = [t.detach().numpy() for t in (Ep, xp, Mp, cp, radius)]
        return torch.from_numpy(O.forward(*a, shape, mpr))

    @staticmethod
    def backward(ctx, g):
        a = [t.detach().numpy() for t in ctx.saved_tensors]
        gE, gX, gM = O.backward(g.detach().numpy(), *a, ctx.mpr)
        return torch.from_numpy(gE), torch.from_numpy(gX), torch.from_numpy(gM), None, None, None, None


def render(h, scene, photons, shape, mpr=20):
    Ep, xp, Mp, cp, radius = RF.receiver_splat_inputs(h, scene, photons)
    return OraclePDS.apply(Ep, xp, Mp, cp, radius, shape, mpr)


def setup(n=24, img=48):
    scene = RF.PlateScene(texel=0.4, receiver_distance=30.0, receiver_half=6.0)
    h = RF.height_field_bumps(n, n, seed=1, bumps=6, amp=(0.0, 0.05), width=(2.0, 5.0))
    t = RF.height_field_bumps(n, n, seed=2, bumps=6, amp=(0.0, 0.05), width=(2.0, 5.0))
    photons = RF.jittered_photons(n, n, scene, per_texel=4, seed=3, smoothing=2.0)
    shape = (1, img, img)
    target = render(t, scene, photons, shape).detach()
    return scene, h, photons, shape, target


def test_photons_land_on_the_receiver_and_energy_is_kept():
    scene, h, photons, shape, target = setup()
    Ep, xp, Mp, cp, radius = RF.receiver_splat_inputs(h, scene, photons)
    assert (xp.abs() < 1).float().mean() > 0.95
    img = render(h, scene, photons, shape)
    # each photon deposits ~ flux * (W/2)(H/2) pixel units when untruncated
    total = float(photons[4].sum()) * shape[1] * shape[2] / 4
    assert 0.5 * total < float(img.sum()) < 1.5 * total


def test_flat_plate_is_a_uniform_splat():
    scene = RF.PlateScene(texel=0.4, receiver_distance=30.0, receiver_half=6.0)
    h = torch.full((24, 24), 1.0, dtype=torch.float64)
    photons = RF.jittered_photons(24, 24, scene, seed=0, smoothing=2.0)
    xy, Du, Dv = RF.trace_to_receiver(h, scene, *photons[:4])
    # normal incidence through parallel faces: straight through, differentials unchanged
    assert torch.allclose(xy[0] * scene.receiver_half, photons[0], atol=1e-12)
    assert torch.allclose(Du[:2] * scene.receiver_half, photons[2][:2], atol=1e-12)


def test_height_gradient_matches_central_differences():
    scene, h, photons, shape, target = setup()
    hv = h.clone().requires_grad_(True)
    img = render(hv, scene, photons, shape)
    loss = 0.5 * ((img - target) ** 2).sum()
    loss.backward()
    grad = hv.grad.detach()
    rng = np.random.default_rng(0)
    idx = [tuple(rng.integers(2, 22, 2)) for _ in range(12)]
    eps = 1e-6

    def L(hh):
        with torch.no_grad():
            return float(0.5 * ((render(hh, scene, photons, shape) - target) ** 2).sum())

    fd, an = [], []
    for (i, j) in idx:
        hp = h.clone(); hp[i, j] += eps
        hm = h.clone(); hm[i, j] -= eps
        fd.append((L(hp) - L(hm)) / (2 * eps))
        an.append(float(grad[i, j]))
    fd, an = np.array(fd), np.array(an)
    assert np.linalg.norm(fd - an) / np.linalg.norm(an) < 1e-4, (fd, an)


def test_config2_gradient_matches_central_differences_on_64_texels():
    """The 256^2 Landweber configuration in full (262,144 photons, 512^2 image): the FP64
    autograd gradient of 0.5 |I - T|^2 against central differences on 64 random texels."""
    import plate_fd as PF
    scene, h, t, photons, du0 = PF.config2()
    target = PF.splat64(t, scene, photons)
    hv = h.clone().requires_grad_(True)
    img = OraclePDS.apply(*RF.receiver_splat_inputs(hv, scene, photons),
                          (1, PF.IMAGE, PF.IMAGE), PF.MPR)
    loss = 0.5 * ((img - torch.from_numpy(target)) ** 2).sum()
    loss.backward()
    # texels whose photons keep their truncation boxes under the +-eps steps (the truncated
    # kernel jumps where a box moves; the derivative is that of the kernel inside its box)
    texels, skipped = PF.smooth_texels(h, scene, photons, 64)
    an = np.array([float(hv.grad[i, j]) for (i, j) in texels])
    fd, smooth = PF.fd_gradient(h, target, scene, photons, texels)
    assert smooth.all() and skipped < 64
    assert np.linalg.norm(fd - an) / np.linalg.norm(an) < 1e-4, (fd, an)


def point_light_setup(n=24, img=48, n_dir=4000, seed=4):
    from oracle import point_light as PLR
    scene = RF.PlateScene(texel=0.4, receiver_distance=30.0, receiver_half=7.0)
    h = RF.height_field_bumps(n, n, seed=seed, bumps=6, amp=(0.0, 0.05), width=(2.0, 5.0))
    half = 0.5 * (n - 1) * scene.texel
    rect = (-half + 0.3, -half + 0.3, half - 0.3, half - 0.3)
    light = (0.4, -0.3, 40.0)
    g = np.random.default_rng(seed)
    u0, u1 = g.random(n_dir), g.random(n_dir)
    d, dt, dp, flux = PLR.point_light(light, rect, 1.0, u0, u1, 6.0, 1.0, 1, 1)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a.T))  # noqa: E731
    return scene, h, light, (T(d), T(dt), T(dp), torch.from_numpy(flux)), (1, img, img)


def test_point_light_trace_hits_the_surface():
    scene, h, light, (d, dt, dp, flux), shape = point_light_setup()
    t, inside = RF.trace_height_field(h, scene, light, d, 1.0)
    p = torch.tensor(light, dtype=torch.float64)[:, None] + t * d
    H, W = h.shape
    fx = p[0] / scene.texel + (W - 1) / 2.0
    fy = p[1] / scene.texel + (H - 1) / 2.0
    hv, _, _ = RF._bilinear(h[None], fx, fy)
    assert bool(inside.all())
    assert float((p[2] - hv[0]).abs().max()) < 1e-12


def test_point_light_height_gradient_matches_central_differences():
    scene, h, light, (d, dt, dp, flux), shape = point_light_setup()

    def render_pl(hh):
        Ep, xp, Mp, cp, radius = RF.point_light_splat_inputs(hh, scene, light, d, dt, dp, flux,
                                                             1.0)
        return OraclePDS.apply(Ep, xp, Mp, cp, radius, shape, 20)

    t2 = RF.height_field_bumps(24, 24, seed=9, bumps=6, amp=(0.0, 0.05), width=(2.0, 5.0))
    target = render_pl(t2).detach()
    hv = h.clone().requires_grad_(True)
    loss = 0.5 * ((render_pl(hv) - target) ** 2).sum()
    loss.backward()
    grad = hv.grad.detach()
    rng = np.random.default_rng(1)
    eps = 1e-7

    def L(hh):
        with torch.no_grad():
            return float(0.5 * ((render_pl(hh) - target) ** 2).sum())

    def boxes(hh):
        with torch.no_grad():
            Ep, xp, Mp, cp, radius = RF.point_light_splat_inputs(hh, scene, light, d, dt, dp,
                                                                 flux, 1.0)
        return O.footprints(xp.numpy(), cp.numpy(), radius.numpy(), shape, 20)[0]

    fd, an = [], []
    while len(fd) < 12:
        i, j = (int(v) for v in rng.integers(3, 21, 2))
        hp = h.clone(); hp[i, j] += eps
        hm = h.clone(); hm[i, j] -= eps
        if not np.array_equal(boxes(hp), boxes(hm)):
            continue  # a truncation box moves: the difference quotient measures a jump
        fd.append((L(hp) - L(hm)) / (2 * eps))
        an.append(float(grad[i, j]))
    fd, an = np.array(fd), np.array(an)
    assert np.linalg.norm(fd - an) / np.linalg.norm(an) < 1e-4, (fd, an)
