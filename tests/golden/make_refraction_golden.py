"""Generates ``refraction_ref.npz``: outputs of the reference's own refraction-chain functions
(pure PyTorch, run here in float64 on the CPU) on seeded inputs.

    python tests/golden/make_refraction_golden.py [--ref-root PATH] [--out FILE]

The reference's ``model`` package is imported from the reference checkout
(``oracle/build_ref.reference_root()``). Its imports that are absent here, or that need a GPU
extension, are replaced by empty stand-in modules before the import: ``PyOptix`` (the OptiX
tracer), ``PhotonDifferentialSplatting`` (the splat extension; its ``pds_forward`` stand-in
records the splat inputs that ``splat_photons`` passes to it and returns a zero image),
``matplotlib`` and ``mpl_toolkits`` (plotting in ``model/utils.py``). The functions called
are unmodified:

  - ``get_normal_from_height_field``  (``model/caustics.py:215-221``)
  - ``refract_reflect_differentials`` (``model/caustics.py:152-212``), with refraction,
    exiting rays (flipped normal) and total internal reflection cases
  - ``Photondifferential._advance_positional_differential``
    (``model/photon_differential.py:69-78``)
  - ``change_of_basis_matrix`` and ``splat_photons`` (``model/caustics.py:224-239``), with
    degenerate photons among them
  - ``fused_silica`` (``model/caustics.py:13-23``)
  - ``slerp``, ``compute_orthonormal_basis``, ``subtended_angle`` (``model/utils.py``) and
    ``compute_point_light_dirs`` (``model/caustics.py:26-70``)
  - the plate's refraction chain composed from the functions above: Sobel normals, the
    bilinear sample of height and normal (``F.grid_sample`` as ``generate_from_point_light``
    samples them, ``model/caustics.py:82-84``; its coordinate derivatives by autograd), the
    transfer onto the tangent plane, the normal derivative (the normalisation of
    ``model/renderable_object.py:400-401``), refraction into the glass, transfer to the flat
    bottom face, refraction out, transfer to the receiver plane and the splat inputs.

Nothing of the reference is copied into this repository: the fixture holds only the seeded
inputs and the reference's outputs.
"""
import argparse
import math
import os
import sys
import types

import numpy as np
import torch
import torch.nn.functional as F

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

CAPTURED = []


def install_stubs():
    popt = types.ModuleType("PyOptix")
    sys.modules["PyOptix"] = popt
    pds = types.ModuleType("PhotonDifferentialSplatting")

    def pds_forward(Ep, xp, Mp, cp, radius, output_size, max_pixel_radius):
        CAPTURED.append(tuple(t.detach().clone() for t in (Ep, xp, Mp, cp, radius)))
        return [torch.zeros(tuple(output_size), dtype=Ep.dtype)]

    def pds_backward(*a):
        raise RuntimeError("not used")

    pds.pds_forward = pds_forward
    pds.pds_backward = pds_backward
    sys.modules["PhotonDifferentialSplatting"] = pds
    mpl = types.ModuleType("matplotlib")
    plt = types.ModuleType("matplotlib.pyplot")
    mpl.pyplot = plt
    sys.modules["matplotlib"] = mpl
    sys.modules["matplotlib.pyplot"] = plt
    tk = types.ModuleType("mpl_toolkits")
    ag = types.ModuleType("mpl_toolkits.axes_grid1")
    ag.ImageGrid = object
    tk.axes_grid1 = ag
    sys.modules["mpl_toolkits"] = tk
    sys.modules["mpl_toolkits.axes_grid1"] = ag


def load_reference(ref_root):
    install_stubs()
    sys.path.insert(0, ref_root)
    import model.caustics as C  # noqa: E402
    import model.photon_differential as P  # noqa: E402
    import model.utils as U  # noqa: E402
    return C, P, U


def unit(v):
    return v / v.norm(dim=-1, keepdim=True)


def bumps(H, W, seed):
    from shapefromcaustics_b200.scene import height_field_bumps
    return height_field_bumps(H, W, seed=seed, bumps=6, base=1.0, amp=(0.0, 0.05),
                              width=(2.0, 5.0))


def case_normals(C, rec):
    h = bumps(24, 20, 1)
    texel = 0.3
    es = torch.tensor([texel, texel], dtype=torch.float64).refine_names("dim")
    hn = h.refine_names("height", "width")
    rec["sobel_h"] = h.numpy()
    rec["sobel_texel"] = np.array(texel)
    rec["sobel_raw"] = C.get_normal_from_height_field(hn, es, normalize=False).rename(None).numpy()
    rec["sobel_unit"] = C.get_normal_from_height_field(hn, es, normalize=True).rename(None).numpy()


def case_refract(C, rec):
    g = torch.Generator().manual_seed(11)
    n = 96
    N = unit(torch.randn((n, 3), generator=g, dtype=torch.float64) * 0.2 +
             torch.tensor([0.0, 0.0, 1.0], dtype=torch.float64))
    d = unit(torch.randn((n, 3), generator=g, dtype=torch.float64) * 0.4 +
             torch.tensor([0.0, 0.0, -1.0], dtype=torch.float64))
    outer = torch.ones(n, dtype=torch.float64)
    inner = torch.full((n,), 1.5, dtype=torch.float64)
    # 16 exiting rays (d.N > 0: the reference flips N and swaps the indices) and 16 rays
    # inside the glass at grazing angles (total internal reflection)
    d[64:80] = -d[64:80]
    t = unit(torch.randn((16, 3), generator=g, dtype=torch.float64))
    graze = unit(N[80:] * 0.2 - t + (t * N[80:]).sum(-1, keepdim=True) * N[80:])
    d[80:] = graze
    outer[80:] = 1.5
    inner[80:] = 1.0
    Dt = torch.randn((n, 3), generator=g, dtype=torch.float64) * 1e-2
    Dp = torch.randn((n, 3), generator=g, dtype=torch.float64) * 1e-2
    dNt = torch.randn((n, 3), generator=g, dtype=torch.float64) * 1e-2
    dNp = torch.randn((n, 3), generator=g, dtype=torch.float64) * 1e-2
    out, Dto, Dpo = C.refract_reflect_differentials(d, N, Dt, Dp, dNt, dNp, outer, inner)
    for k, v in dict(d=d, N=N, Dt=Dt, Dp=Dp, dNt=dNt, dNp=dNp, outer=outer, inner=inner,
                     out=out, Dt_out=Dto, Dp_out=Dpo).items():
        rec["refract_" + k] = v.numpy()


def case_transfer(P, rec):
    g = torch.Generator().manual_seed(12)
    n = 64
    nm = ("sample", "dim")
    normal = unit(torch.randn((n, 3), generator=g, dtype=torch.float64) * 0.3 +
                  torch.tensor([0.0, 0.0, 1.0], dtype=torch.float64))
    direction = unit(torch.randn((n, 3), generator=g, dtype=torch.float64) * 0.3 -
                     torch.tensor([0.0, 0.0, 1.0], dtype=torch.float64))
    Du, Dv, Dt, Dp = (torch.randn((n, 3), generator=g, dtype=torch.float64) * 0.1
                      for _ in range(4))
    length = torch.rand(n, generator=g, dtype=torch.float64) * 5
    pd = P.Photondifferential(normal=normal.refine_names(*nm), direction=direction.refine_names(*nm),
                              Du=Du.refine_names(*nm), Dv=Dv.refine_names(*nm),
                              Dtheta=Dt.refine_names(*nm), Dphi=Dp.refine_names(*nm),
                              length=length.refine_names("sample"))
    pd._advance_positional_differential()
    for k, v in dict(normal=normal, direction=direction, Du=Du, Dv=Dv, Dt=Dt, Dp=Dp,
                     length=length).items():
        rec["transfer_" + k] = v.numpy()
    rec["transfer_Du_out"] = pd.Du.rename(None).numpy()
    rec["transfer_Dv_out"] = pd.Dv.rename(None).numpy()


def splat_inputs_ref(C, P, Du, Dv, normal, flux, channel, xy):
    """The reference's splat_photons on [3, N] differentials; -> its pds_forward inputs."""
    pd = P.Photondifferential(Du=Du, Dv=Dv, shading_normal=normal, flux=flux,
                              channel_coords=channel)
    CAPTURED.clear()
    C.splat_photons(pd, xy, (1, 8, 8), max_pixel_radius=20)
    return CAPTURED[-1]


def case_splat_inputs(C, P, rec):
    g = torch.Generator().manual_seed(13)
    n = 80
    Du = torch.randn((3, n), generator=g, dtype=torch.float64) * 0.01
    Dv = torch.randn((3, n), generator=g, dtype=torch.float64) * 0.01
    Du[2] = 0
    Dv[2] = 0
    Dv[:, 5] = 2.0 * Du[:, 5]     # degenerate: parallel differentials
    Dv[:, 17] = 0.0               # degenerate: zero differential
    normal = torch.zeros((3, n), dtype=torch.float64)
    normal[2] = 1.0
    flux = torch.rand(n, generator=g, dtype=torch.float64)
    channel = torch.randint(0, 3, (n,), generator=g)
    xy = torch.rand((2, n), generator=g, dtype=torch.float64) * 2 - 1
    Ep, xp, Mp, cp, radius = splat_inputs_ref(C, P, Du, Dv, normal, flux, channel, xy)
    for k, v in dict(Du=Du, Dv=Dv, normal=normal, flux=flux, channel=channel, xy=xy, Ep=Ep,
                     xp=xp, Mp=Mp, cp=cp, radius=radius).items():
        rec["splat_" + k] = v.numpy()


def case_dispersion(C, rec):
    lam = np.linspace(0.40, 0.70, 31)
    rec["silica_lambda_um"] = lam
    rec["silica_n"] = np.array([C.fused_silica(float(v)) for v in lam])


def case_point_light(C, U, rec):
    # compute_point_light_dirs over a 6 x 5 grid of surface coordinates, seeded
    H, W, inner, sims, smooth = 6, 5, 2, 3, 5.0
    xs = torch.linspace(-1.0, 1.0, W, dtype=torch.float64)
    ys = torch.linspace(-0.8, 0.8, H, dtype=torch.float64)
    coords = torch.stack(torch.meshgrid(xs, ys, indexing="xy")).refine_names("dim", "height", "width")
    light = torch.tensor([0.1, -0.2, 10.0], dtype=torch.float64).refine_names("dim")
    torch.manual_seed(5)
    pd = C.compute_point_light_dirs(1.0, 1, light, coords, num_simul=sims, num_inner_simul=inner,
                                    smoothing=smooth, energy=1e-5)
    torch.manual_seed(5)
    coeffs = torch.rand(2, H, W * inner, dtype=torch.float64)
    rec["plight_coords"] = coords.rename(None).numpy()
    rec["plight_light"] = light.rename(None).numpy()
    rec["plight_params"] = np.array([1.0, 1, sims, inner, smooth, 1e-5])
    rec["plight_coeffs"] = coeffs.numpy()
    rec["plight_direction"] = pd.direction.rename(None).numpy()
    rec["plight_Dtheta"] = pd.Dtheta.rename(None).numpy()
    rec["plight_Dphi"] = pd.Dphi.rename(None).numpy()
    rec["plight_flux"] = pd.flux.rename(None).numpy()
    rec["plight_position"] = pd.position.rename(None).numpy()
    # the helpers on their own
    g = torch.Generator().manual_seed(14)
    p0 = unit(torch.randn((40, 3), generator=g, dtype=torch.float64))
    p1 = unit(p0 + 0.3 * torch.randn((40, 3), generator=g, dtype=torch.float64))
    tt = torch.rand((40, 1), generator=g, dtype=torch.float64)
    rec["slerp_p0"], rec["slerp_p1"], rec["slerp_t"] = p0.numpy(), p1.numpy(), tt.numpy()
    rec["slerp_out"] = U.slerp(p0, p1, tt).numpy()
    nrm = unit(torch.randn((3, 40), generator=g, dtype=torch.float64))
    nrm[:, 0] = torch.tensor([0.0, 0.0, -1.0], dtype=torch.float64)  # the basis' singular case
    b1, b2 = U.compute_orthonormal_basis(nrm.refine_names("dim", "sample"), dim="dim")
    rec["onb_n"], rec["onb_b1"], rec["onb_b2"] = nrm.numpy(), b1.rename(None).numpy(), b2.rename(None).numpy()


def case_plate_chain(C, P, rec):
    """The plate's chain from reference functions, for collimated light on a height field."""
    H = W = 16
    texel, ior, dist, half = 0.4, 1.5, 30.0, 6.0
    light = unit(torch.tensor([0.03, -0.02, -1.0], dtype=torch.float64))
    h = bumps(H, W, 3)
    g = torch.Generator().manual_seed(15)
    per = 2
    n = (H - 2) * (W - 2) * per
    iy = torch.arange(1, H - 1, dtype=torch.float64).repeat_interleave((W - 2) * per)
    ix = torch.arange(1, W - 1, dtype=torch.float64).repeat_interleave(per).repeat(H - 2)
    px = (ix + torch.rand(n, generator=g, dtype=torch.float64) - 0.5 - (W - 1) / 2.0) * texel
    py = (iy + torch.rand(n, generator=g, dtype=torch.float64) - 0.5 - (H - 1) / 2.0) * texel
    # photons in float32 (what the CUDA kernels take), evaluated in float64
    px, py = px.float().double(), py.float().double()
    du0 = 0.05
    flux = torch.full((n,), 1.0 / n, dtype=torch.float64)
    es = torch.tensor([texel, texel], dtype=torch.float64).refine_names("dim")
    Nfield = C.get_normal_from_height_field(h.refine_names("height", "width"), es,
                                            normalize=False).rename(None)
    # bilinear samples with texel centres at integers (align_corners=True), border clamp
    gx = (px / texel) * (2.0 / (W - 1))
    gy = (py / texel) * (2.0 / (H - 1))
    grid = torch.stack((gx, gy), -1).reshape(1, 1, n, 2).requires_grad_(True)
    field = torch.cat((h[None], Nfield), 0)[None]
    samp = F.grid_sample(field, grid, mode="bilinear", padding_mode="border",
                         align_corners=True)[0, :, 0, :]  # [4, n]
    ddx, ddy = [], []
    for c in range(4):
        (gr,) = torch.autograd.grad(samp[c].sum(), grid, retain_graph=True)
        ddx.append(gr[0, 0, :, 0] * (2.0 / ((W - 1) * texel)))
        ddy.append(gr[0, 0, :, 1] * (2.0 / ((H - 1) * texel)))
    samp = samp.detach()
    hz = samp[0]
    Nt = samp[1:].t()                                  # [n, 3] un-normalised normal
    dNdx = torch.stack(ddx[1:], 0).t().detach()        # [n, 3]
    dNdy = torch.stack(ddy[1:], 0).t().detach()
    d = light[None].expand(n, 3).contiguous()
    nu = unit(Nt)
    nm = ("sample", "dim")

    def transfer(D, Dd, length, normal, dirn):
        pd = P.Photondifferential(normal=normal.refine_names(*nm), direction=dirn.refine_names(*nm),
                                  Du=D.refine_names(*nm), Dv=D.clone().refine_names(*nm),
                                  Dtheta=Dd.refine_names(*nm), Dphi=Dd.clone().refine_names(*nm),
                                  length=length.refine_names("sample"))
        pd._advance_positional_differential()
        return pd.Du.rename(None)

    zero = torch.zeros((n, 3), dtype=torch.float64)
    Du0 = torch.zeros((n, 3), dtype=torch.float64)
    Dv0 = torch.zeros((n, 3), dtype=torch.float64)
    Du0[:, 0] = du0
    Dv0[:, 1] = du0
    Du1 = transfer(Du0, zero, torch.zeros(n, dtype=torch.float64), nu, d)
    Dv1 = transfer(Dv0, zero, torch.zeros(n, dtype=torch.float64), nu, d)
    ndn = (Nt * Nt).sum(-1, keepdim=True)

    def dunit(dN):
        return (ndn * dN - (Nt * dN).sum(-1, keepdim=True) * Nt) / ndn ** 1.5

    dnu = dunit(dNdx * Du1[:, :1] + dNdy * Du1[:, 1:2])
    dnv = dunit(dNdx * Dv1[:, :1] + dNdy * Dv1[:, 1:2])
    one = torch.ones(n, dtype=torch.float64)
    t1, Ddu, Ddv = C.refract_reflect_differentials(d, nu, zero, zero, dnu, dnv, one, one * ior)
    p1 = torch.stack((px, py, hz), -1)
    s1 = -p1[:, 2] / t1[:, 2]
    p2 = p1 + s1[:, None] * t1
    ez = torch.zeros((n, 3), dtype=torch.float64)
    ez[:, 2] = 1.0
    Du2 = transfer(Du1, Ddu, s1, ez, t1)
    Dv2 = transfer(Dv1, Ddv, s1, ez, t1)
    t2, Ddu2, Ddv2 = C.refract_reflect_differentials(t1, ez, Ddu, Ddv, zero, zero, one * ior, one)
    s2 = (-dist - p2[:, 2]) / t2[:, 2]
    p3 = p2 + s2[:, None] * t2
    Du3 = transfer(Du2, Ddu2, s2, ez, t2) / half
    Dv3 = transfer(Dv2, Ddv2, s2, ez, t2) / half
    xy = (p3[:, :2] / half).t().contiguous()
    Ep, xp, Mp, cp, radius = splat_inputs_ref(C, P, Du3.t().contiguous(), Dv3.t().contiguous(),
                                              ez.t().contiguous(), flux,
                                              torch.zeros(n, dtype=torch.int64), xy)
    rec["chain_h"] = h.numpy()
    rec["chain_params"] = np.array([texel, ior, dist, half, du0])
    rec["chain_light"] = light.numpy()
    rec["chain_px"], rec["chain_py"], rec["chain_flux"] = px.numpy(), py.numpy(), flux.numpy()
    for k, v in dict(Ep=Ep, xp=xp, Mp=Mp, cp=cp, radius=radius).items():
        rec["chain_" + k] = v.numpy()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=None)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                  "refraction_ref.npz"))
    a = ap.parse_args()
    from oracle import build_ref
    ref_root = a.ref_root or build_ref.reference_root()
    if ref_root is None:
        raise SystemExit("no reference checkout (set PDS_REFERENCE_ROOT)")
    C, P, U = load_reference(ref_root)
    rec = {}
    case_normals(C, rec)
    case_refract(C, rec)
    case_transfer(P, rec)
    case_splat_inputs(C, P, rec)
    case_dispersion(C, rec)
    case_point_light(C, U, rec)
    case_plate_chain(C, P, rec)
    np.savez_compressed(a.out, **rec)
    print("wrote", a.out, len(rec), "arrays")


if __name__ == "__main__":
    main()
