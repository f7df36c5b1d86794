"""FP64 restatement of the refraction-to-receiver chain for a height-field glass plate.
TEST INFRASTRUCTURE ONLY: the tests use it as the float64 reference of the fused refraction
kernels (``pds_refract_forward_f32`` / ``pds_refract_backward_f32``); the product never imports
it. Its building blocks are pinned to the reference's own functions by the fixture
``tests/golden/refraction_ref.npz`` (``tests/golden/make_refraction_golden.py``).

The differentiable step between a height field and the splat inputs, for collimated light
falling on the plate (the analytic height-field case the reference's OptiX tracer handles for
this scene). Per photon:

  1. surface sample: bilinear height and bilinear (unnormalised) Sobel normal at a jittered
     position; the Sobel normal field follows ``get_normal_from_height_field``
     (``model/caustics.py:215-221``: replicate padding, kernel scaled by -1/(8 texel)).
  2. positional-differential transfer onto the surface (Frisvad 2014,
     ``model/photon_differential.py:69-78``): ``D' = D - (n.D)/(n.d) d + t (Dd - (n.Dd)/(n.d) d)``.
  3. Snell refraction of the direction and of its differentials (Igehy 1999,
     ``model/caustics.py:152-212``): with ``cosi = d.N``, ``eta``,
     ``k = 1 - eta^2 (1 - cosi^2)``, ``coso = eta cosi + sqrt(k)``,
     ``d' = eta d - coso N`` and
     ``Dd' = eta Dd - (coso dN + (eta - eta^2 cosi / -sqrt(k)) (Dd.N + d.dN) N)``;
     a ray leaving the denser side (``d.N > 0``) swaps the indices and flips the normal, and
     ``k <= 0`` reflects (``d - 2 (d.N) N``, Igehy's reflection differentials), as the
     reference does; the normal derivative ``dN`` along the positional differential uses
     ``(|N|^2 dN~ - (N.dN~) N) / |N|^3`` of the un-normalised normal ``N~``
     (``model/renderable_object.py:391-401``).
  4. propagation inside the glass to the flat bottom face (z = 0), refraction out
     (flat face: ``dN = 0``), propagation to the receiver plane ``z = -receiver_distance``.
  5. receiver coordinates normalised by the receiver half-extent, and the splat inputs of
     ``model/caustics.py:224-239`` (``change_of_basis_matrix``, ``splat_photons``).

The normal derivative is taken along the photon's whole positional differential at the hit
(position and direction parts). The reference passes only the direction-induced part
(``model/caustics.py:271`` uses ``Dtheta_hit``), which is the whole differential for its
point light (Du = Dv = 0 at the first hit) but is zero for collimated light.

Units: millimetres. Everything is written over tensors of any float dtype, so the same code
runs in float64 on the CPU (the finite-difference reference) and float32 on the GPU.
"""
import math

import torch
import torch.nn.functional as F

from shapefromcaustics_b200.scene import PlateScene, height_field_bumps  # noqa: F401

__all__ = ["PlateScene", "sobel_normals", "sample_surface", "trace_to_receiver",
           "height_field_bumps", "jittered_photons", "splat_inputs", "refract_differentials",
           "transfer"]


def sobel_normals(h, texel):
    """Un-normalised normal field ``[3, H, W]`` = (-dh/dx, -dh/dy, 1) by the Sobel operator."""
    k = torch.tensor([[[[-1, 0, 1], [-2, 0, 2], [-1, 0, 1]]],
                      [[[-1, -2, -1], [0, 0, 0], [1, 2, 1]]]], dtype=h.dtype, device=h.device)
    k = k * (-1.0 / (8.0 * texel))
    g = F.conv2d(F.pad(h[None, None], (1, 1, 1, 1), mode="replicate"), k)[0]
    return torch.cat((g, torch.ones_like(h)[None]), dim=0)


def _bilinear(field, fx, fy):
    """Bilinear sample of ``field [C, H, W]`` at continuous texel coordinates (texel centres
    at integers, clamped to the border) -> values ``[C, N]`` and d/dfx, d/dfy ``[C, N]``."""
    C, H, W = field.shape
    fx = fx.clamp(0, W - 1)
    fy = fy.clamp(0, H - 1)
    x0 = fx.detach().floor().clamp(max=W - 2).long() if W > 1 else torch.zeros_like(fx, dtype=torch.long)
    y0 = fy.detach().floor().clamp(max=H - 2).long() if H > 1 else torch.zeros_like(fy, dtype=torch.long)
    x1 = (x0 + 1).clamp(max=W - 1)
    y1 = (y0 + 1).clamp(max=H - 1)
    ax = fx - x0
    ay = fy - y0
    flat = field.reshape(C, -1)
    v00 = flat[:, y0 * W + x0]
    v01 = flat[:, y0 * W + x1]
    v10 = flat[:, y1 * W + x0]
    v11 = flat[:, y1 * W + x1]
    top = v00 + (v01 - v00) * ax
    bot = v10 + (v11 - v10) * ax
    val = top + (bot - top) * ay
    ddx = (v01 - v00) * (1 - ay) + (v11 - v10) * ay
    ddy = bot - top
    return val, ddx, ddy


def sample_surface(h, scene, px, py):
    """Surface point, un-normalised normal and its spatial derivatives at world (px, py)."""
    H, W = h.shape
    fx = px / scene.texel + (W - 1) / 2.0
    fy = py / scene.texel + (H - 1) / 2.0
    N = sobel_normals(h, scene.texel)
    hv, hdx, hdy = _bilinear(h[None], fx, fy)
    nv, ndx, ndy = _bilinear(N, fx, fy)
    return hv[0], nv, ndx / scene.texel, ndy / scene.texel


def _dot(a, b):
    return (a * b).sum(0)


def transfer(D, Dd, t, n, d):
    """Positional differential D with direction differential Dd carried along direction d for
    length t onto a plane of normal n (``model/photon_differential.py:69-78``: the hit's
    positional part ``D - (n.D)/(n.d) d`` plus ``t (Dd - (n.Dd)/(n.d) d)``)."""
    nd = _dot(n, d)
    return D - _dot(n, D) / nd * d + t * (Dd - _dot(n, Dd) / nd * d)


_transfer = transfer


def refract_differentials(d, N, Dd, dN, n_outer, n_inner):
    """Direction and direction differential after refraction (or total internal reflection)
    at unit normal N with normal derivative dN, ``model/caustics.py:152-212``:
    ``cosi = clamp(d.N, -1, 1)``; where ``cosi > 0`` the indices swap and N, dN flip sign
    (``cosi`` itself keeps its sign, as in the reference); ``eta = n_i / n_t``,
    ``k = 1 - eta^2 (1 - cosi^2)``; ``k > 0`` refracts (Igehy 1999, p. 4), otherwise the ray
    reflects, ``d - 2 cosi N`` with ``Dd - 2 (cosi dN + (Dd.N + d.dN) N)`` (p. 3).
    Vectors are ``[3, N]``; ``n_outer``, ``n_inner`` scalars or ``[N]``."""
    cosi = _dot(d, N).clamp(-1, 1)
    flip = cosi > 0
    no = torch.as_tensor(n_outer, dtype=d.dtype, device=d.device).expand_as(cosi)
    ni = torch.as_tensor(n_inner, dtype=d.dtype, device=d.device).expand_as(cosi)
    etai = torch.where(flip, ni, no)
    etat = torch.where(flip, no, ni)
    sgn = torch.where(flip, -torch.ones_like(cosi), torch.ones_like(cosi))
    Nf = sgn * N
    dNf = sgn * dN
    eta = etai / etat
    k = 1 - eta * eta * (1 - cosi * cosi)
    rm = k > 0
    neg_sq = -torch.sqrt(torch.where(rm, k, torch.ones_like(k)))
    coso = eta * cosi - neg_sq
    dn_term = _dot(Dd, Nf) + _dot(d, dNf)
    out_r = eta * d - coso * Nf
    Dout_r = eta * Dd - (coso * dNf + ((eta - eta * eta * cosi / neg_sq) * dn_term) * Nf)
    out_l = d - 2 * cosi * Nf
    Dout_l = Dd - 2 * (cosi * dNf + dn_term * Nf)
    return torch.where(rm, out_r, out_l), torch.where(rm, Dout_r, Dout_l)


def _refract(d, N, Dd, dN, eta):
    """Refraction at unit normal N facing the incident side (d.N < 0) with index ratio eta."""
    return refract_differentials(d, N, Dd, dN, eta, 1.0)


def change_of_basis_matrix(Du, Dv, normal):
    """``model/caustics.py:224-230``: ``Mp = 2 / (Du.(Dv x n)) [Dv x n ; n x Du]`` (2 x 3 x N)
    and the non-degenerate mask (denominator != 0); degenerate photons get a finite
    placeholder here instead of being dropped."""
    tmp = torch.cross(Dv, normal, dim=0)
    den = (Du * tmp).sum(0)
    good = den != 0
    factor = 2.0 / torch.where(good, den, torch.ones_like(den))
    return factor * torch.stack((tmp, torch.cross(normal, Du, dim=0)), dim=0), good


def splat_inputs(Du, Dv, normal, flux, channel):
    """Splat inputs ``(Ep, Mp, cp, radius)`` of ``model/caustics.py:233-239``:
    ``radius = 0.5 max(|Du|, |Dv|)``, ``Ep = 4 flux / |Du x Dv|``; degenerate photons keep
    their slot with channel -1 (the splat skips them)."""
    Mp, good = change_of_basis_matrix(Du, Dv, normal)
    radius = 0.5 * torch.maximum(Du.norm(dim=0), Dv.norm(dim=0))
    area = torch.cross(Du, Dv, dim=0).norm(dim=0)
    Ep = flux / torch.where(good, area, torch.ones_like(area)) * 4
    cp = torch.where(good, channel, torch.full_like(channel, -1)).reshape(1, -1)
    return Ep.contiguous(), Mp.contiguous(), cp.contiguous(), radius.contiguous()


def _unit_normal_and_derivative(Nt, dNt):
    """n = N~/|N~| and its derivative along a differential (``renderable_object.py:391-401``)."""
    ndn = _dot(Nt, Nt)
    n = Nt / torch.sqrt(ndn)
    dn = (ndn * dNt - _dot(Nt, dNt) * Nt) / ndn ** 1.5
    return n, dn


def trace_to_receiver(h, scene, px, py, Du0, Dv0):
    """Per-photon receiver position (normalised, ``[2, N]``) and receiver-plane positional
    differentials ``Du, Dv [3, N]`` (normalised units) for collimated photons entering the
    plate's top surface at world (px, py) with initial positional differentials Du0, Dv0
    ``[3, N]`` (in the plane perpendicular to the light)."""
    dt = h.dtype
    dev = h.device
    n_ph = px.shape[0]
    d = torch.tensor(scene.light_dir, dtype=dt, device=dev)[:, None].expand(3, n_ph)
    zero = torch.zeros((3, n_ph), dtype=dt, device=dev)
    hz, Nt, Ntx, Nty = sample_surface(h, scene, px, py)
    # 1. onto the top surface: the photon crosses the surface at its sample point; carry the
    #    source plane differentials onto the local tangent plane
    Ntn = Nt / torch.sqrt(_dot(Nt, Nt))
    Du1 = _transfer(Du0, zero, 0.0, Ntn, d)
    Dv1 = _transfer(Dv0, zero, 0.0, Ntn, d)
    dNu = Ntx * Du1[0] + Nty * Du1[1]
    dNv = Ntx * Dv1[0] + Nty * Dv1[1]
    n, dnu = _unit_normal_and_derivative(Nt, dNu)
    _, dnv = _unit_normal_and_derivative(Nt, dNv)
    # 2. refraction air -> glass at the top face (normal points up, against the light)
    eta = 1.0 / scene.ior
    t1, Ddu = _refract(d, n, zero, dnu, eta)
    _, Ddv = _refract(d, n, zero, dnv, eta)
    p1 = torch.stack((px, py, hz))
    # 3. to the bottom face z = 0
    s1 = -p1[2] / t1[2]
    p2 = p1 + s1 * t1
    nz = torch.zeros_like(zero)
    nz[2] = 1.0
    Du2 = _transfer(Du1, Ddu, s1, nz, t1)
    Dv2 = _transfer(Dv1, Ddv, s1, nz, t1)
    # 4. refraction glass -> air at the flat bottom face (normal facing the glass side: +z)
    t2, Ddu2 = _refract(t1, nz, Ddu, zero, scene.ior)
    _, Ddv2 = _refract(t1, nz, Ddv, zero, scene.ior)
    # 5. to the receiver plane z = -receiver_distance
    s2 = (-scene.receiver_distance - p2[2]) / t2[2]
    p3 = p2 + s2 * t2
    Du3 = _transfer(Du2, Ddu2, s2, nz, t2)
    Dv3 = _transfer(Dv2, Ddv2, s2, nz, t2)
    inv = 1.0 / scene.receiver_half
    return p3[:2] * inv, Du3 * inv, Dv3 * inv


def jittered_photons(H, W, scene, per_texel=4, seed=0, smoothing=4.0, dtype=torch.float64,
                     device="cpu"):
    """Collimated photons: ``per_texel`` uniformly jittered entry points per texel, with
    initial positional differentials ``2 smoothing sqrt(A / (pi N))`` along x and y (the
    reference scales its light's differentials the same way, ``model/caustics.py:60-61``)
    and flux 1/N. Returns ``(px, py, Du0, Dv0, flux)``."""
    g = torch.Generator(device="cpu").manual_seed(int(seed))
    n = H * W * per_texel
    iy = torch.arange(H, dtype=torch.float64).repeat_interleave(W * per_texel)
    ix = torch.arange(W, dtype=torch.float64).repeat_interleave(per_texel).repeat(H)
    jx = torch.rand(n, generator=g, dtype=torch.float64) - 0.5
    jy = torch.rand(n, generator=g, dtype=torch.float64) - 0.5
    px = (ix + jx - (W - 1) / 2.0) * scene.texel
    py = (iy + jy - (H - 1) / 2.0) * scene.texel
    area = H * W * scene.texel ** 2
    scale = 2.0 * smoothing * math.sqrt(area / (math.pi * n))
    Du0 = torch.zeros((3, n), dtype=torch.float64)
    Dv0 = torch.zeros((3, n), dtype=torch.float64)
    Du0[0] = scale
    Dv0[1] = scale
    flux = torch.full((n,), 1.0 / n, dtype=torch.float64)
    cast = dict(dtype=dtype, device=device)
    return px.to(**cast), py.to(**cast), Du0.to(**cast), Dv0.to(**cast), flux.to(**cast)


def receiver_splat_inputs(h, scene, photons, channel=None):
    """Splat inputs ``(Ep, xp, Mp, cp, radius)`` of the plate for the given photons."""
    px, py, Du0, Dv0, flux = photons
    xy, Du, Dv = trace_to_receiver(h, scene, px, py, Du0, Dv0)
    nrm = torch.zeros_like(Du)
    nrm[2] = 1.0
    if channel is None:
        channel = torch.zeros(px.shape[0], dtype=torch.int64, device=px.device)
    Ep, Mp, cp, radius = splat_inputs(Du, Dv, nrm, flux, channel)
    return Ep, xy.contiguous(), Mp, cp, radius


def trace_height_field(h, scene, origin, d, plane_z, iterations=12):
    """Ray parameter t of the first hit of rays ``origin + t d`` (``origin [3]``, ``d [3, N]``
    unit, pointing down) with the bilinear height-field surface ``z = h(x, y)``: Newton steps on
    ``f(t) = o_z + t d_z - h(o_xy + t d_xy)`` from the plane ``z = plane_z`` (the height field is
    assumed to have no overhangs and no occluding bump before the hit, as the reference's
    ``generate_from_point_light`` assumes for its samples). Differentiable in ``h``: at the
    converged root the Newton map's derivative is the implicit one, ``dt/dh = w / f'(t)``.
    -> (t [N], inside [N] bool: the hit lies over the field)."""
    H, W = h.shape
    o = torch.as_tensor(origin, dtype=h.dtype, device=h.device)[:, None]
    t = (o[2] - plane_z) / (-d[2])
    for _ in range(iterations):
        p = o + t * d
        fx = p[0] / scene.texel + (W - 1) / 2.0
        fy = p[1] / scene.texel + (H - 1) / 2.0
        hv, hdx, hdy = _bilinear(h[None], fx, fy)
        f = p[2] - hv[0]
        fp = d[2] - (hdx[0] * d[0] + hdy[0] * d[1]) / scene.texel
        t = t - f / fp
    p = o + t * d
    fx = p[0] / scene.texel + (W - 1) / 2.0
    fy = p[1] / scene.texel + (H - 1) / 2.0
    inside = (fx >= 0) & (fx <= W - 1) & (fy >= 0) & (fy <= H - 1)
    return t, inside


def trace_point_light_to_receiver(h, scene, origin, d, Dth, Dph, plane_z):
    """Receiver position (normalised, ``[2, N]``) and receiver-plane differentials ``[3, N]``
    of point-light photons (``origin``, unit directions ``d [3, N]``, direction differentials
    ``Dth, Dph [3, N]``): the traced hit on the height field, the positional differentials
    carried from the light to the hit (``model/photon_differential.py:69-78`` with ``Du = Dv =
    0`` at the light), refraction into the glass with the direction differentials, the flat
    bottom face and the receiver plane as in ``trace_to_receiver``. -> (xy, Du, Dv, inside)."""
    dt = h.dtype
    n_ph = d.shape[1]
    zero = torch.zeros((3, n_ph), dtype=dt, device=h.device)
    t, inside = trace_height_field(h, scene, origin, d, plane_z)
    o = torch.as_tensor(origin, dtype=dt, device=h.device)[:, None]
    p1 = o + t * d
    _, Nt, Ntx, Nty = sample_surface(h, scene, p1[0], p1[1])
    Ntn = Nt / torch.sqrt(_dot(Nt, Nt))
    Du1 = transfer(zero, Dth, t, Ntn, d)
    Dv1 = transfer(zero, Dph, t, Ntn, d)
    dNu = Ntx * Du1[0] + Nty * Du1[1]
    dNv = Ntx * Dv1[0] + Nty * Dv1[1]
    n, dnu = _unit_normal_and_derivative(Nt, dNu)
    _, dnv = _unit_normal_and_derivative(Nt, dNv)
    t1, Ddu = _refract(d, n, Dth, dnu, 1.0 / scene.ior)
    _, Ddv = _refract(d, n, Dph, dnv, 1.0 / scene.ior)
    s1 = -p1[2] / t1[2]
    p2 = p1 + s1 * t1
    nz = torch.zeros_like(zero)
    nz[2] = 1.0
    Du2 = transfer(Du1, Ddu, s1, nz, t1)
    Dv2 = transfer(Dv1, Ddv, s1, nz, t1)
    t2, Ddu2 = _refract(t1, nz, Ddu, zero, scene.ior)
    _, Ddv2 = _refract(t1, nz, Ddv, zero, scene.ior)
    s2 = (-scene.receiver_distance - p2[2]) / t2[2]
    p3 = p2 + s2 * t2
    Du3 = transfer(Du2, Ddu2, s2, nz, t2)
    Dv3 = transfer(Dv2, Ddv2, s2, nz, t2)
    inv = 1.0 / scene.receiver_half
    return p3[:2] * inv, Du3 * inv, Dv3 * inv, inside


def point_light_splat_inputs(h, scene, origin, d, Dth, Dph, flux, plane_z, channel=None):
    """Splat inputs ``(Ep, xp, Mp, cp, radius)`` of point-light photons; photons whose hit
    misses the field get channel -1."""
    xy, Du, Dv, inside = trace_point_light_to_receiver(h, scene, origin, d, Dth, Dph, plane_z)
    nrm = torch.zeros_like(Du)
    nrm[2] = 1.0
    if channel is None:
        channel = torch.zeros(d.shape[1], dtype=torch.int64, device=d.device)
    channel = torch.where(inside, channel, torch.full_like(channel, -1))
    Ep, Mp, cp, radius = splat_inputs(Du, Dv, nrm, flux, channel)
    return Ep, xy.contiguous(), Mp, cp, radius
