"""Central finite differences of the Landweber step's loss in float64, for the gradient
checks of the 256^2 configuration (test helper, not collected by pytest).

Configuration: a 256 x 256 height field (1 mm base plus 32 Gaussian bumps, amplitude
U[0, 50] um, width U[4, 24] texels), collimated light at normal incidence, 4 jittered photons
per texel (262,144), n = 1.5, receiver 50 mm below, 512 x 512 image, loss
L = 0.5 |I - T|^2 against the image of a second seeded field.

The loss is evaluated with the FP64 refraction chain (``oracle/refraction_chain.py``) and the
FP64 oracle splat. A texel's height moves only the photons whose bilinear sample or Sobel
stencil reads it (entry points within two texels), so L(h +- eps e_ij) is formed from the
image of all photons by replacing those photons' contribution: exact, and fast enough for 64
texels of the full configuration.
"""
import math

import numpy as np
import torch

from oracle import oracle as O
from oracle import refraction_chain as RC
from shapefromcaustics_b200.scene import PlateScene, height_field_bumps

N_FIELD, IMAGE, PER_TEXEL, MPR = 256, 512, 4, 20
TEXEL, DIST = 0.1, 50.0


def config2(seed=0):
    """-> scene, h (float64), target field (float64), photons (float64 values of float32
    entry points: px, py, Du0, Dv0, flux), du0."""
    half = 0.5 * N_FIELD * TEXEL * 1.1
    scene = PlateScene(texel=TEXEL, ior=1.5, receiver_distance=DIST, receiver_half=half)
    h = height_field_bumps(N_FIELD, N_FIELD, seed=seed, bumps=32, base=1.0, amp=(0.0, 0.05),
                           width=(4.0, 24.0))
    t = height_field_bumps(N_FIELD, N_FIELD, seed=seed + 1, bumps=32, base=1.0, amp=(0.0, 0.05),
                           width=(4.0, 24.0))
    # float32-exact values (the CUDA path takes float32 fields and entry points)
    h = h.float().double()
    t = t.float().double()
    px, py, Du0, Dv0, flux = RC.jittered_photons(N_FIELD, N_FIELD, scene, per_texel=PER_TEXEL,
                                                 seed=seed + 2, smoothing=1.0)
    du0 = 3.0 * 2.0 * half / IMAGE  # 3-pixel initial footprint
    Du0[0] = du0
    Dv0[1] = du0
    px, py, flux = px.float().double(), py.float().double(), flux.float().double()
    return scene, h, t, (px, py, Du0, Dv0, flux), du0


def splat64(h, scene, photons, shape=(1, IMAGE, IMAGE)):
    a = [x.detach().numpy() for x in RC.receiver_splat_inputs(h, scene, photons)]
    return O.forward(*a, shape, MPR)


def texel_photons(i, j, per_texel=PER_TEXEL, n=N_FIELD):
    """Indices of the photons whose entry texel lies within two texels of (i, j)."""
    rows = np.arange(max(i - 2, 0), min(i + 3, n))
    cols = np.arange(max(j - 2, 0), min(j + 3, n))
    tex = (rows[:, None] * n + cols[None, :]).reshape(-1)
    return (tex[:, None] * per_texel + np.arange(per_texel)[None, :]).reshape(-1)


def footprints(h, scene, photons, shape=(1, IMAGE, IMAGE)):
    """The reference's integer footprint (centre pixel, radii) of each photon."""
    Ep, xp, Mp, cp, radius = RC.receiver_splat_inputs(h, scene, photons)
    f, _ = O.footprints(xp.detach().numpy(), cp.numpy(), radius.detach().numpy(), shape, MPR)
    return f


def fd_gradient(h, target_img, scene, photons, texels, eps=1e-7):
    """Central differences of L = 0.5 |I - T|^2 at the given texels -> (values, smooth).

    The reference's footprint is truncated to a box of integer radii around an integer centre
    pixel, so the loss jumps where a photon's box moves; ``smooth[k]`` is False where some
    photon moved by texel k changes its box between h - eps and h + eps (the difference
    quotient then measures the jump, not the derivative)."""
    full = splat64(h, scene, photons)
    out, smooth = [], []
    for (i, j) in texels:
        idx = torch.from_numpy(texel_photons(i, j))
        sub = tuple(x[..., idx] for x in photons)
        base = splat64(h, scene, sub)
        vals, boxes = [], []
        for s in (1.0, -1.0):
            hp = h.clone()
            hp[i, j] += s * eps
            img = full - base + splat64(hp, scene, sub)
            vals.append(0.5 * float(np.sum((img - target_img) ** 2)))
            boxes.append(footprints(hp, scene, sub))
        out.append((vals[0] - vals[1]) / (2 * eps))
        smooth.append(bool(np.array_equal(boxes[0], boxes[1])))
    return np.array(out), np.array(smooth)


def random_texels(k=64, seed=0, margin=3, n=N_FIELD):
    rng = np.random.default_rng(seed)
    return [tuple(int(v) for v in rng.integers(margin, n - margin, 2)) for _ in range(k)]


def smooth_texels(h, scene, photons, k=64, seed=0, eps=1e-7, margin=3, n=N_FIELD):
    """k random texels whose photons keep their footprint boxes under +-eps (drawn until k are
    found; -> texels, number of texels skipped)."""
    rng = np.random.default_rng(seed)
    got, skipped = [], 0
    while len(got) < k:
        i, j = (int(v) for v in rng.integers(margin, n - margin, 2))
        idx = torch.from_numpy(texel_photons(i, j))
        sub = tuple(x[..., idx] for x in photons)
        b = []
        for s in (1.0, -1.0):
            hp = h.clone()
            hp[i, j] += s * eps
            b.append(footprints(hp, scene, sub))
        if np.array_equal(b[0], b[1]):
            got.append((i, j))
        else:
            skipped += 1
    return got, skipped
