"""Projected Landweber update of the height field and the reconstruction loop around it.

``landweber_update`` is the fused device update (``pds_landweber_update_f32``) of the
reference's PyTorch ops (``shape_from_caustics.py:184-189`` extShrink, ``:228-241``
VconsHeur, ``:386-398`` the update). ``reconstruct`` runs the reference's pixel-basis Landweber loop
(``optimization_loop_landweber_pixel``, ``:343-420``) for a height-field plate on the
sm_100a kernels: simulate (refraction + splat), L2 discrepancy against the target image,
backward to the height field, update.
"""
import ctypes
from dataclasses import dataclass

import torch

from . import _lib
from ._lib import check, lib
from .splatting import _ptr, _stream

__all__ = ["LandweberParams", "landweber_update", "reconstruct"]


@dataclass
class LandweberParams:
    tau: float = 1e-1          # tau_pixel
    alpha: float = 2e-3        # alpha_pixel (shrink threshold = tau * alpha)
    lower: float = 0.0
    upper: float = 0.3
    d1: float = 1.0
    d2: float = 1.0
    gamma: float = 0.1
    radius: int = 2            # volume_radius

    def c_struct(self):
        p = _lib.PdsLandweber()
        p.tau = self.tau
        p.shrink = self.tau * self.alpha
        p.lower = self.lower
        p.upper = self.upper
        p.d1 = self.d1
        p.d2 = self.d2
        p.gamma = self.gamma
        p.radius = int(self.radius)
        return p


def landweber_update(d, grad, mask, params, workspace=None):
    """In-place fused update of the height-field offset ``d [H, W]`` (float32, device)."""
    for t, nm in ((d, "d"), (grad, "grad"), (mask, "mask")):
        if not (t.is_cuda and t.is_contiguous() and t.dtype == torch.float32 and t.shape == d.shape):
            raise RuntimeError(f"{nm} must be a contiguous float32 CUDA tensor shaped like d")
    rows, cols = d.shape
    nbytes = lib().pds_landweber_workspace_bytes(rows, cols)
    if workspace is None or workspace.numel() < nbytes:
        workspace = torch.empty(int(nbytes), dtype=torch.uint8, device=d.device)
    p = params.c_struct()
    with torch.cuda.device(d.device):
        check(lib().pds_landweber_update_f32(_ptr(d), _ptr(grad), _ptr(mask), rows, cols,
                                             ctypes.byref(p), _ptr(workspace), workspace.numel(),
                                             _stream(d.device)))
    return d


def render_plate(height, scene, px, py, flux, params, shape, max_pixel_radius=20):
    """Caustic image of the plate (no gradient)."""
    from .plate import PlateSplat
    with torch.no_grad():
        return PlateSplat.apply(height, px, py, flux, params, shape, max_pixel_radius, False)


def photon_source(H, W, per_texel, texel, seed, offset, device, out=None):
    """Entry points of ``per_texel`` uniformly jittered photons per texel from the device
    source (``pds_photon_source_f32``: Philox4x32-10 keyed by ``seed``, counter blocks from
    ``offset``, two photons a block; photon i in texel i % (H W)). Returns ``(px, py, next_offset)``; passing
    ``next_offset`` to the next call draws a disjoint stream. ``out``: optional ``(px, py)``
    float32 device tensors of ``H * W * per_texel`` elements to write into."""
    n = H * W * per_texel
    if out is not None:
        px, py = out
        if px.numel() != n or py.numel() != n:
            raise RuntimeError(f"out must hold {n} photons")
    else:
        px = torch.empty(n, dtype=torch.float32, device=device)
        py = torch.empty(n, dtype=torch.float32, device=device)
    with torch.cuda.device(px.device):
        check(lib().pds_photon_source_f32(H, W, per_texel, float(texel), int(seed) & (2 ** 64 - 1),
                                          int(offset), _ptr(px), _ptr(py), _stream(px.device)))
    return px, py, int(offset) + (n + 1) // 2


def jitter(H, W, scene, per_texel, generator, device):
    """Entry points of ``per_texel`` uniformly jittered photons per texel, on the device:
    ``per_texel`` samples of one photon per texel in raster order (photon i in texel
    i % (H W)), like the device source."""
    n = H * W * per_texel
    idx = torch.arange(n, device=device)
    texel = idx % (H * W)
    iy = (texel // W).float()
    ix = (texel % W).float()
    j = torch.rand((2, n), generator=generator, device=device) - 0.5
    px = (ix + j[0] - (W - 1) / 2.0) * scene.texel
    py = (iy + j[1] - (H - 1) / 2.0) * scene.texel
    return px.contiguous(), py.contiguous()


def reconstruct(h_true, base, scene, iterations=200, sims=16, per_texel=4, image=1024,
                footprint_px=3.0, params=None, mask=None, seed=0, keep_plan=True, target=None,
                log_every=0, objective="l2_sq"):
    """The reference's pixel-basis Landweber loop (``shape_from_caustics.py:343-420``,
    default options) for a height-field plate, all on the device.

    Each iteration splats ``sims`` simulations of ``per_texel`` freshly jittered photons
    per texel into one image (the reference's sum over simulations, ``:351-353``), takes the
    data term against the target, back-propagates to the height-field offset through the splat
    and refraction kernels and applies the fused projected update. ``keep_plan``: the splat
    plan and the refracted splat inputs are kept from forward to backward (about 120 B per
    photon held); False recomputes both in the backward. ``objective``: ``"l2_sq"`` is the reference's data term
    ``0.5 |I - T|^2`` (``hyperparameter_helper.py:29-30``, its default ``--data_norm``), for
    which ``params.tau`` is the reference's ``tau_pixel``; ``"normalized"`` divides it by
    ``|T|^2``. The logged discrepancy is the reference's ``sqrt(2 fdis) / |T|``
    (``shape_from_caustics.py:363``) either way. ``footprint_px`` sets the photons' initial
    positional differentials to that many receiver pixels (the reference's splat smoothing,
    ``model/caustics.py:60-61``). Returns a dict with the reconstructed offset, the
    per-iteration discrepancy and height RMSE."""
    from .plate import PlateSplat, plate_params
    if objective not in ("l2_sq", "normalized"):
        raise ValueError("objective must be 'l2_sq' or 'normalized'")
    dev = h_true.device
    H, W = h_true.shape
    n = H * W * per_texel * sims
    du0 = footprint_px * 2.0 * scene.receiver_half / image
    pp = plate_params(scene, du0)
    shape = (1, image, image)
    flux = torch.full((n,), 1.0 / n, device=dev)
    d_true = h_true - base
    offset = 0
    if target is None:
        px, py, offset = photon_source(H, W, per_texel * sims, scene.texel, seed, offset, dev)
        target = render_plate(h_true, scene, px, py, flux, pp, shape)
    tnorm2 = float((target * target).sum())
    scale = 1.0 if objective == "l2_sq" else 1.0 / tnorm2
    if params is None:
        vol = float(d_true.sum())
        params = LandweberParams(d1=0.75 * vol, d2=1.25 * vol)
    if mask is None:
        mask = torch.ones_like(h_true)
    d = torch.zeros_like(h_true)
    ws = torch.empty(int(lib().pds_landweber_workspace_bytes(H, W)), dtype=torch.uint8, device=dev)
    hist = {"discrepancy": [], "rmse": []}
    logged = []
    for it in range(iterations):
        px, py, offset = photon_source(H, W, per_texel * sims, scene.texel, seed, offset, dev)
        hv = (base + d).requires_grad_(True)
        img = PlateSplat.apply(hv, px, py, flux, pp, shape, 20, keep_plan)
        diff = img - target
        fdis = 0.5 * (diff * diff).sum()
        (fdis * scale).backward()
        landweber_update(d, hv.grad, mask, params, ws)
        if log_every and (it % log_every == 0 or it == iterations - 1):
            # kept on the device (no synchronisation inside the loop), read after it
            logged.append((it, (2.0 * fdis.detach()).sqrt() / tnorm2 ** 0.5,
                           ((d - d_true) ** 2).mean().sqrt()))
    for it, dis, err in logged:
        hist["discrepancy"].append((it, float(dis)))
        hist["rmse"].append((it, float(err)))
    rmse = float(((d - d_true) ** 2).mean().sqrt())
    return {"d": d, "rmse": rmse, "history": hist, "target": target, "photons_per_iteration": n}


def iteration_phases(base, target, scene, d, mask, params, sims=16, per_texel=4, image=1024,
                     footprint_px=3.0, seed=0, offset=0, objective="l2_sq", reps=3,
                     keep_plan=True):
    """CUDA-event times (ms, median of ``reps``) of the phases of one Landweber iteration of
    ``reconstruct``, run phase by phase on the current stream: photon source, refraction
    forward, plan, splat forward, data-term gradient, (with ``keep_plan`` False: the
    refraction and the plan recomputed for the backward,) splat backward, refraction backward,
    update. The height field is ``base + d``; ``d`` is updated in place."""
    import statistics
    from .plate import plate_params, refract_backward_planned, refract_forward
    from .splatting import SplatPlan
    dev = d.device
    H, W = d.shape
    n = H * W * per_texel * sims
    pp = plate_params(scene, footprint_px * 2.0 * scene.receiver_half / image)
    shape = (1, image, image)
    flux = torch.full((n,), 1.0 / n, device=dev)
    ws = torch.empty(int(lib().pds_landweber_workspace_bytes(H, W)), dtype=torch.uint8, device=dev)
    scale = 1.0 if objective == "l2_sq" else 1.0 / float((target * target).sum())
    names = ["source", "refract_fwd", "plan", "splat_fwd", "data_grad", "recompute",
             "splat_bwd", "refract_bwd", "update"]
    times = {k: [] for k in names}
    for r in range(reps + 1):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(names) + 1)]
        ev[0].record()
        px, py, offset = photon_source(H, W, per_texel * sims, scene.texel, seed, offset, dev)
        ev[1].record()
        hv = (base + d).contiguous()
        Ep, xp, Mp, cp, radius = refract_forward(hv, px, py, flux, pp)
        ev[2].record()
        plan = SplatPlan(Ep, xp, Mp, cp, radius, shape, 20)
        ev[3].record()
        img = plan.forward()
        ev[4].record()
        g_img = ((img - target) * scale).contiguous()
        ev[5].record()
        if not keep_plan:
            plan = SplatPlan(*refract_forward(hv, px, py, flux, pp), shape, 20)
        ev[6].record()
        plan.backward(g_img, records=True)
        ev[7].record()
        gh = refract_backward_planned(hv, px, py, flux, pp, plan)
        ev[8].record()
        landweber_update(d, gh, mask, params, ws)
        ev[9].record()
        torch.cuda.synchronize()
        if r > 0:
            for k, name in enumerate(names):
                times[name].append(ev[k].elapsed_time(ev[k + 1]))
    out = {k: statistics.median(v) for k, v in times.items()}
    if keep_plan:
        del out["recompute"]
    out["total"] = sum(out.values())
    return out
