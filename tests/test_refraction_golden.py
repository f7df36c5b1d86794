"""The FP64 refraction chain of the oracle (``oracle/refraction_chain.py``) and the product's
splat-input builder and dispersion formula, pinned to the reference's own functions: the
fixture ``tests/golden/refraction_ref.npz`` holds their outputs on seeded inputs
(``tests/golden/make_refraction_golden.py``: ``get_normal_from_height_field``,
``refract_reflect_differentials``, ``_advance_positional_differential``,
``change_of_basis_matrix`` / ``splat_photons``, ``fused_silica``, the point light's helpers, and
the plate's chain composed from them). All comparisons are float64 against float64.
"""
import os

import numpy as np
import pytest
import torch

from oracle import refraction_chain as RC

GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                            "refraction_ref.npz"))
TOL = 1e-12


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def t(name):
    return torch.from_numpy(GOLD[name])


def test_sobel_normals_equal_get_normal_from_height_field():
    n = RC.sobel_normals(t("sobel_h"), float(GOLD["sobel_texel"]))
    assert rel(n, GOLD["sobel_raw"]) < TOL
    unit = n / n.norm(dim=0, keepdim=True)
    assert rel(unit, GOLD["sobel_unit"]) < TOL


def test_refraction_equals_refract_reflect_differentials():
    # rows are samples in the fixture ([N, 3]); the chain works on [3, N]
    d, N = t("refract_d").t(), t("refract_N").t()
    outs = []
    for D, dN in (("refract_Dt", "refract_dNt"), ("refract_Dp", "refract_dNp")):
        outs.append(RC.refract_differentials(d, N, t(D).t(), t(dN).t(), t("refract_outer"),
                                             t("refract_inner")))
    assert rel(outs[0][0].t(), GOLD["refract_out"]) < TOL
    assert rel(outs[0][1].t(), GOLD["refract_Dt_out"]) < TOL
    assert rel(outs[1][1].t(), GOLD["refract_Dp_out"]) < TOL
    # each regime on its own: refraction (0-63), exiting rays (64-79), total reflection (80-95)
    for sl in (slice(0, 64), slice(64, 80), slice(80, 96)):
        assert rel(outs[0][1].t()[sl], GOLD["refract_Dt_out"][sl]) < TOL


def test_transfer_equals_advance_positional_differential():
    args = dict(n=t("transfer_normal").t(), d=t("transfer_direction").t(),
                t=t("transfer_length"))
    Du = RC.transfer(t("transfer_Du").t(), t("transfer_Dt").t(), args["t"], args["n"], args["d"])
    Dv = RC.transfer(t("transfer_Dv").t(), t("transfer_Dp").t(), args["t"], args["n"], args["d"])
    assert rel(Du.t(), GOLD["transfer_Du_out"]) < TOL
    assert rel(Dv.t(), GOLD["transfer_Dv_out"]) < TOL


@pytest.mark.parametrize("impl", ["oracle", "product"])
def test_splat_inputs_equal_splat_photons(impl):
    if impl == "oracle":
        fn = RC.splat_inputs
    else:
        from shapefromcaustics_b200.caustics import splat_inputs as fn
    Ep, Mp, cp, radius = fn(t("splat_Du"), t("splat_Dv"), t("splat_normal"), t("splat_flux"),
                            t("splat_channel"))
    good = cp[0] >= 0
    # the reference drops degenerate photons (Du . (Dv x n) == 0); here they keep their slot
    # with channel -1
    assert int((~good).sum()) == 2 and not bool(good[5]) and not bool(good[17])
    assert rel(Ep[good], GOLD["splat_Ep"]) < TOL
    assert rel(Mp[:, :, good], GOLD["splat_Mp"]) < TOL
    assert rel(radius[good], GOLD["splat_radius"]) < TOL
    assert np.array_equal(cp[:, good].numpy(), GOLD["splat_cp"])
    assert np.array_equal(t("splat_xy")[:, good].numpy(), GOLD["splat_xp"])


def test_plate_chain_equals_the_reference_functions_composed():
    texel, ior, dist, half, du0 = (float(v) for v in GOLD["chain_params"])
    scene = RC.PlateScene(texel=texel, ior=ior, receiver_distance=dist, receiver_half=half,
                          light_dir=tuple(GOLD["chain_light"]))
    n = GOLD["chain_px"].shape[0]
    Du0 = torch.zeros((3, n), dtype=torch.float64)
    Dv0 = torch.zeros((3, n), dtype=torch.float64)
    Du0[0] = du0
    Dv0[1] = du0
    photons = (t("chain_px"), t("chain_py"), Du0, Dv0, t("chain_flux"))
    Ep, xp, Mp, cp, radius = RC.receiver_splat_inputs(t("chain_h"), scene, photons)
    assert bool((cp >= 0).all())
    assert rel(xp, GOLD["chain_xp"]) < 1e-10
    assert rel(Ep, GOLD["chain_Ep"]) < 1e-10
    assert rel(Mp, GOLD["chain_Mp"]) < 1e-10
    assert rel(radius, GOLD["chain_radius"]) < 1e-10


def test_fused_silica_dispersion_equals_the_reference():
    from shapefromcaustics_b200.scene import fused_silica
    lam = GOLD["silica_lambda_um"]
    n = np.array([fused_silica(float(v)) for v in lam])
    assert rel(n, GOLD["silica_n"]) < 1e-15
    # over the visible range the index falls from about 1.470 to 1.456
    assert 1.45 < n.min() < n.max() < 1.48 and np.all(np.diff(n) < 0)
    # tensors too
    nt = fused_silica(torch.from_numpy(lam))
    assert rel(nt.numpy(), GOLD["silica_n"]) < 1e-15


def point_light_case():
    coords = GOLD["plight_coords"]
    plane_z, nwl, sims, inner, smooth, energy = (float(v) for v in GOLD["plight_params"])
    rect = (coords[0].min(), coords[1].min(), coords[0].max(), coords[1].max())
    coeffs = GOLD["plight_coeffs"].reshape(2, -1)
    return GOLD["plight_light"], rect, plane_z, coeffs, smooth, energy, int(sims), int(inner)


def test_point_light_restatement_equals_compute_point_light_dirs():
    from oracle import point_light as PLR
    light, rect, z, coeffs, smooth, energy, sims, inner = point_light_case()
    d, dt, dp, flux = PLR.point_light(light, rect, z, coeffs[0], coeffs[1], smooth, energy, sims,
                                      inner)
    assert rel(d, GOLD["plight_direction"]) < TOL
    assert rel(dt, GOLD["plight_Dtheta"]) < TOL
    assert rel(dp, GOLD["plight_Dphi"]) < TOL
    assert rel(flux, GOLD["plight_flux"]) < TOL
    # the helpers on their own
    assert rel(PLR.slerp(GOLD["slerp_p0"], GOLD["slerp_p1"], GOLD["slerp_t"]), GOLD["slerp_out"]) < TOL
    b1, b2 = PLR.onb(GOLD["onb_n"].T)
    assert rel(b1.T, GOLD["onb_b1"]) < TOL and rel(b2.T, GOLD["onb_b2"]) < TOL
