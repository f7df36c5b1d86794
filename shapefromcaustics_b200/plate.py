"""Height field -> caustic image on the receiver, differentiable in the height field, on the
fused sm_100a refraction kernels and the splat kernels.

``PlateSplat.apply(height, photons, plate, output_size, max_pixel_radius)`` is the
refraction-to-receiver step followed by the splat (``model/caustics.py:242-291`` for this
scene, with ``splat_photons`` ``:233-239`` at its end). The backward runs the splat backward
and then the refraction backward kernel, which recomputes each photon's path from the height
field: refracted positions and differentials are never stored, and with
``keep_plan=False`` neither is the splat's binning, so the memory held between the passes is
the height field and the photons' entry points (12 bytes per photon).

``photons`` is ``(px, py, flux)`` (``[N]`` each, float32, device) plus an optional channel
``[N]`` int64; ``plate`` a ``PlateScene`` (``scene.py``) with ``du0``, the initial
positional differential length.
"""
import ctypes

import torch

from . import _lib
from ._lib import check, lib
from .splatting import SplatPlan, _ptr, _stream

__all__ = ["PlateParams", "plate_params", "refract_forward", "refract_backward", "PlateSplat",
           "PointLight", "point_light", "point_light_source", "refract_point_forward",
           "refract_point_backward", "PointPlateSplat", "BatchedPlate", "BatchedPlateSplat"]


PlateParams = _lib.PdsPlate


def plate_params(scene, du0):
    """``pds_plate`` of a ``PlateScene`` with initial differential length ``du0``."""
    p = PlateParams()
    p.texel = scene.texel
    p.ior = scene.ior
    p.receiver_distance = scene.receiver_distance
    p.receiver_half = scene.receiver_half
    for k in range(3):
        p.light_dir[k] = scene.light_dir[k]
    p.du0 = float(du0)
    return p


def _fn(name):
    return getattr(lib(), name)


def _check_f32(t, name):
    if not (t.is_cuda and t.is_contiguous() and t.dtype == torch.float32):
        raise RuntimeError(f"{name} must be a contiguous float32 CUDA tensor")


def refract_forward(height, px, py, flux, params, channel=None):
    """Splat inputs ``(Ep, xp, Mp, cp, radius)`` of the photons (``pds_refract_forward_f32``)."""
    for t, nm in ((height, "height"), (px, "px"), (py, "py"), (flux, "flux")):
        _check_f32(t, nm)
    n = px.numel()
    dev = height.device
    Ep = torch.empty(n, device=dev)
    xp = torch.empty((2, n), device=dev)
    Mp = torch.empty((2, 3, n), device=dev)
    cp = torch.empty((1, n), dtype=torch.int64, device=dev)
    radius = torch.empty(n, device=dev)
    with torch.cuda.device(dev):
        check(_fn("pds_refract_forward_f32")(
            _ptr(height), height.shape[0], height.shape[1], ctypes.byref(params), _ptr(px),
            _ptr(py), _ptr(flux), _ptr(channel) if channel is not None else None, n, _ptr(Ep),
            _ptr(xp), _ptr(Mp), _ptr(cp), _ptr(radius), _stream(dev)))
    return Ep, xp, Mp, cp, radius


def refract_backward(height, px, py, flux, params, gE, gX, gM, grad_height=None):
    """Adds d L / d height for splat-input gradients (``pds_refract_backward_f32``)."""
    n = px.numel()
    if grad_height is None:
        grad_height = torch.zeros_like(height)
    with torch.cuda.device(height.device):
        check(_fn("pds_refract_backward_f32")(
            _ptr(height), height.shape[0], height.shape[1], ctypes.byref(params), _ptr(px),
            _ptr(py), _ptr(flux), n, _ptr(gE.contiguous()), _ptr(gX.contiguous()),
            _ptr(gM.contiguous()), _ptr(grad_height), _stream(height.device)))
    return grad_height


def refract_backward_planned(height, px, py, flux, params, plan, grad_height=None):
    """Adds d L / d height from the gradient records that ``plan.backward(g, records=True)``
    left in the plan's workspace (``pds_refract_backward_planned_f32``): the refraction
    backward without the gradients' spread into grad_Ep / grad_xp / grad_Mp. ``plan`` is the
    ``SplatPlan`` of these photons' refracted splat inputs."""
    n = px.numel()
    if grad_height is None:
        grad_height = torch.zeros_like(height)
    with torch.cuda.device(height.device):
        check(_fn("pds_refract_backward_planned_f32")(
            _ptr(height), height.shape[0], height.shape[1], ctypes.byref(params), _ptr(px),
            _ptr(py), _ptr(flux), n, plan.C, plan.H, plan.W, _ptr(plan.ws), plan.ws.numel(),
            ctypes.byref(plan.cfg), _ptr(grad_height), _stream(height.device)))
    return grad_height


class PlateSplat(torch.autograd.Function):
    """Caustic image of a height-field plate; differentiable in the height field."""

    @staticmethod
    def forward(ctx, height, px, py, flux, params, output_size, max_pixel_radius, keep_plan=True):
        h = height.detach().contiguous()
        Ep, xp, Mp, cp, radius = refract_forward(h, px, py, flux, params)
        plan = SplatPlan(Ep, xp, Mp, cp, radius, output_size, max_pixel_radius)
        img = plan.forward()
        ctx.save_for_backward(h, px, py, flux)
        ctx.params = params
        ctx.shape = tuple(int(v) for v in output_size)
        ctx.mpr = int(max_pixel_radius)
        # keep_plan: the plan and the refracted splat inputs are kept for the backward (the
        # reference's PDS saves its inputs, model/photon_differential.py:10); otherwise both
        # are recomputed there (less memory: 12 B per photon held instead of about 120 B)
        ctx.plan_ws = plan.ws if keep_plan else None
        ctx.inputs = (Ep, xp, Mp, cp, radius) if keep_plan else None
        ctx.cfg = plan.cfg
        return img

    @staticmethod
    def backward(ctx, grad_img):
        h, px, py, flux = ctx.saved_tensors
        if ctx.inputs is not None:
            Ep, xp, Mp, cp, radius = ctx.inputs
        else:
            Ep, xp, Mp, cp, radius = refract_forward(h, px, py, flux, ctx.params)
        if ctx.plan_ws is not None:
            plan = SplatPlan.__new__(SplatPlan)
            plan.n = Ep.numel()
            plan.C, plan.H, plan.W = ctx.shape
            plan.mpr = ctx.mpr
            plan.cfg = ctx.cfg
            plan.device = h.device
            plan.inputs = (Ep, xp, Mp, cp, radius)
            plan.ws = ctx.plan_ws
        else:
            plan = SplatPlan(Ep, xp, Mp, cp, radius, ctx.shape, ctx.mpr, config=ctx.cfg)
        # the splat gradients stay in the plan's workspace as records, read there by the
        # refraction backward
        plan.backward(grad_img.contiguous(), records=True)
        gh = refract_backward_planned(h, px, py, flux, ctx.params, plan)
        ctx.plan_ws = None
        ctx.inputs = None
        return gh, None, None, None, None, None, None, None


PointLight = _lib.PdsPointLight


def point_light(position, rect, plane_z, smoothing, energy, simulations=1, inner=1,
                wavelengths=1):
    """``pds_point_light`` of a light at ``position`` whose photons spread over
    ``rect = (xmin, ymin, xmax, ymax)`` on the plane ``z = plane_z`` (the reference's
    ``compute_point_light_dirs`` arguments: smoothing, energy, num_simul, num_inner_simul and
    the number of wavelengths)."""
    L = PointLight()
    for k in range(3):
        L.position[k] = float(position[k])
    L.plane_z = float(plane_z)
    L.xmin, L.ymin, L.xmax, L.ymax = (float(v) for v in rect)
    L.smoothing = float(smoothing)
    L.energy = float(energy)
    L.simulations = int(simulations)
    L.inner = int(inner)
    L.wavelengths = int(wavelengths)
    return L


def point_light_source(light, n_directions, device, seed=0, offset=0, coeffs=None):
    """Photon directions of a point light on the device (``pds_point_light_source_f32``):
    ``(direction [3, n], dtheta [3, n], dphi [3, n], flux [n], next_offset)`` with
    ``n = n_directions * light.wavelengths``. The two uniform numbers of each direction come
    from ``coeffs [2, n_directions]`` (float32, device) when given, else from the Philox
    source keyed by ``seed`` at counter ``offset``; ``next_offset`` draws a disjoint stream."""
    n = int(n_directions) * int(light.wavelengths)
    dev = torch.device(device)
    out = [torch.empty((3, n), device=dev) for _ in range(3)] + [torch.empty(n, device=dev)]
    if coeffs is not None:
        _check_f32(coeffs, "coeffs")
        if tuple(coeffs.shape) != (2, int(n_directions)):
            raise RuntimeError("coeffs must be [2, n_directions]")
    with torch.cuda.device(dev):
        check(_fn("pds_point_light_source_f32")(
            ctypes.byref(light), int(n_directions), int(seed) & (2 ** 64 - 1), int(offset),
            _ptr(coeffs) if coeffs is not None else None, *(_ptr(t) for t in out), _stream(dev)))
    return (*out, int(offset) + (int(n_directions) + 1) // 2)


def refract_point_forward(height, light, params, direction, dtheta, dphi, flux, channel=None):
    """Splat inputs ``(Ep, xp, Mp, cp, radius)`` of point-light photons traced onto the plate
    (``pds_refract_point_forward_f32``)."""
    for t, nm in ((height, "height"), (direction, "direction"), (dtheta, "dtheta"),
                  (dphi, "dphi"), (flux, "flux")):
        _check_f32(t, nm)
    n = flux.numel()
    dev = height.device
    Ep = torch.empty(n, device=dev)
    xp = torch.empty((2, n), device=dev)
    Mp = torch.empty((2, 3, n), device=dev)
    cp = torch.empty((1, n), dtype=torch.int64, device=dev)
    radius = torch.empty(n, device=dev)
    with torch.cuda.device(dev):
        check(_fn("pds_refract_point_forward_f32")(
            _ptr(height), height.shape[0], height.shape[1], ctypes.byref(params),
            ctypes.byref(light), _ptr(direction), _ptr(dtheta), _ptr(dphi), _ptr(flux),
            _ptr(channel) if channel is not None else None, n, _ptr(Ep), _ptr(xp), _ptr(Mp),
            _ptr(cp), _ptr(radius), _stream(dev)))
    return Ep, xp, Mp, cp, radius


def refract_point_backward(height, light, params, direction, dtheta, dphi, flux, gE, gX, gM,
                           grad_height=None):
    """Adds d L / d height for point-light photons (``pds_refract_point_backward_f32``)."""
    n = flux.numel()
    if grad_height is None:
        grad_height = torch.zeros_like(height)
    with torch.cuda.device(height.device):
        check(_fn("pds_refract_point_backward_f32")(
            _ptr(height), height.shape[0], height.shape[1], ctypes.byref(params),
            ctypes.byref(light), _ptr(direction), _ptr(dtheta), _ptr(dphi), _ptr(flux), n,
            _ptr(gE.contiguous()), _ptr(gX.contiguous()), _ptr(gM.contiguous()),
            _ptr(grad_height), _stream(height.device)))
    return grad_height


class PointPlateSplat(torch.autograd.Function):
    """Caustic image of the plate lit by a point light (photons traced onto the height-field
    surface); differentiable in the height field. ``photons`` = ``(direction, dtheta, dphi,
    flux)`` as from ``point_light_source``."""

    @staticmethod
    def forward(ctx, height, direction, dtheta, dphi, flux, light, params, output_size,
                max_pixel_radius):
        h = height.detach().contiguous()
        inputs = refract_point_forward(h, light, params, direction, dtheta, dphi, flux)
        plan = SplatPlan(*inputs, output_size, max_pixel_radius)
        img = plan.forward()
        ctx.save_for_backward(h, direction, dtheta, dphi, flux)
        ctx.light, ctx.params = light, params
        ctx.shape = tuple(int(v) for v in output_size)
        ctx.mpr = int(max_pixel_radius)
        ctx.cfg = plan.cfg
        return img

    @staticmethod
    def backward(ctx, grad_img):
        h, direction, dtheta, dphi, flux = ctx.saved_tensors
        inputs = refract_point_forward(h, ctx.light, ctx.params, direction, dtheta, dphi, flux)
        plan = SplatPlan(*inputs, ctx.shape, ctx.mpr, config=ctx.cfg)
        gE, gX, gM = plan.backward(grad_img.contiguous())
        gh = refract_point_backward(h, ctx.light, ctx.params, direction, dtheta, dphi, flux, gE,
                                    gX, gM)
        return gh, None, None, None, None, None, None, None, None


class BatchedPlate:
    """Many simulations of one height-field plate in one launch sequence: each simulation has
    its own photon count, image size and plate parameters (light direction, the refractive
    index of its wavelength, initial differential length), and all share the height field.

    ``sims`` is a list of ``(n_photons, (C, H, W), pds_plate)``; photons are the simulations'
    entry points concatenated in order. The forward refracts every photon in one batched launch
    (``pds_batch_refract_forward_f32``) and splats all simulations through one plan and one
    forward (``BatchedSplat``); the backward runs the batched splat backward, leaving its
    gradients as records in the plan's workspace, and one batched refraction backward that
    reads them there into the height field's gradient. ``keep_inputs``: the refracted splat
    inputs of the forward are kept for the backward (as the reference's PDS saves them);
    False recomputes them there (48 B per photon less held between the passes). The reference
    runs its simulations one after another and sums them (``shape_from_caustics.py:351-353``);
    ``images(flat)`` gives the per-simulation images."""

    def __init__(self, sims, max_pixel_radius, device, config=None, keep_inputs=True):
        from .splatting import BatchedSplat
        self.splat = BatchedSplat([(n, shape) for n, shape, _ in sims], max_pixel_radius,
                                  device, config=config)
        self.device = self.splat.device
        n_sims = len(sims)
        table = (PlateParams * n_sims)()
        begins = []
        b = 0
        for k, (n, _, p) in enumerate(sims):
            ctypes.memmove(ctypes.byref(table, k * ctypes.sizeof(PlateParams)), ctypes.byref(p),
                           ctypes.sizeof(PlateParams))
            begins.append(b)
            b += int(n)
        self.n_sims = n_sims
        self.n_total = b
        self.plates_dev = torch.frombuffer(bytearray(bytes(table)), dtype=torch.uint8).to(
            self.device)
        self.begins_dev = torch.tensor(begins, dtype=torch.int64, device=self.device)
        self.image_elems = self.splat.image_elems
        self.keep_inputs = bool(keep_inputs)

    def _inputs(self, height, px, py, flux):
        n = self.n_total
        if px.numel() != n or py.numel() != n or flux.numel() != n:
            raise RuntimeError(f"batch expects {n} photons")
        for t, nm in ((height, "height"), (px, "px"), (py, "py"), (flux, "flux")):
            _check_f32(t, nm)
        dev = self.device
        Ep = torch.empty(n, device=dev)
        xp = torch.empty((2, n), device=dev)
        Mp = torch.empty((2, 3, n), device=dev)
        cp = torch.empty((1, n), dtype=torch.int64, device=dev)
        radius = torch.empty(n, device=dev)
        with torch.cuda.device(dev):
            check(_fn("pds_batch_refract_forward_f32")(
                _ptr(height), height.shape[0], height.shape[1], _ptr(self.plates_dev),
                _ptr(self.begins_dev), self.n_sims, _ptr(px), _ptr(py), _ptr(flux), None, n,
                _ptr(Ep), _ptr(xp), _ptr(Mp), _ptr(cp), _ptr(radius), _stream(dev)))
        return Ep, xp, Mp, cp, radius

    def forward(self, height, px, py, flux, out=None):
        """Flat images of all simulations (plans the splat; keeps the plan for backward)."""
        inputs = self._inputs(height, px, py, flux)
        self.splat.plan(*inputs)
        img = self.splat.forward(out)
        if not self.keep_inputs:
            self.splat.inputs = None
        return img

    def backward(self, height, px, py, flux, grad_flat, grad_height=None):
        """Adds d L / d height for the flat images' gradient (after ``forward`` on the same
        height field and photons)."""
        if not self.keep_inputs or self.splat.inputs is None:
            self.splat.inputs = self._inputs(height, px, py, flux)
        # the splat gradients stay in the plan's workspace as records, read there by the
        # batched refraction backward
        self.splat.backward(grad_flat, records=True)
        if not self.keep_inputs:
            self.splat.inputs = None
        if grad_height is None:
            grad_height = torch.zeros_like(height)
        sp = self.splat
        with torch.cuda.device(self.device):
            check(_fn("pds_batch_refract_backward_planned_f32")(
                _ptr(height), height.shape[0], height.shape[1], _ptr(self.plates_dev),
                _ptr(self.begins_dev), self.n_sims, _ptr(px), _ptr(py), _ptr(flux),
                self.n_total, sp.n_tiles, _ptr(sp.ws), sp.ws.numel(), ctypes.byref(sp.cfg),
                _ptr(grad_height), _stream(self.device)))
        return grad_height

    def images(self, flat):
        return self.splat.images(flat)


class BatchedPlateSplat(torch.autograd.Function):
    """Flat images of a ``BatchedPlate``'s simulations; differentiable in the height field."""

    @staticmethod
    def forward(ctx, height, px, py, flux, batch):
        h = height.detach().contiguous()
        img = batch.forward(h, px, py, flux)
        ctx.save_for_backward(h, px, py, flux)
        ctx.batch = batch
        return img

    @staticmethod
    def backward(ctx, grad_flat):
        h, px, py, flux = ctx.saved_tensors
        gh = ctx.batch.backward(h, px, py, flux, grad_flat.contiguous())
        return gh, None, None, None, None
