"""Fused refraction-to-receiver kernels (pds_refract_*_f32) against the float64 PyTorch
refraction chain (itself checked by central finite differences in test_refraction.py), and
the end-to-end differentiable plate (PlateSplat) against the FP64 chain + FP64 oracle splat.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import refraction_chain as RF

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def scene_and_photons(n=64, seed=0, smoothing=3.0):
    scene = RF.PlateScene(texel=0.4, receiver_distance=30.0, receiver_half=14.0)
    h = RF.height_field_bumps(n, n, seed=seed, bumps=10, base=1.0, amp=(0.0, 0.05),
                              width=(2.0, 8.0)).float()
    ph = RF.jittered_photons(n, n, scene, per_texel=4, seed=seed + 1, smoothing=smoothing)
    du0 = float(ph[2][0, 0])
    return scene, h, ph, du0


def torch_inputs64(h, scene, ph):
    px, py, Du0, Dv0, flux = (t.double() for t in ph)
    return RF.receiver_splat_inputs(h.double(), scene, (px.float().double(), py.float().double(),
                                                        Du0, Dv0, flux.float().double()))


def test_refract_forward_matches_float64_chain(cuda):
    from shapefromcaustics_b200 import plate as PL
    scene, h, ph, du0 = scene_and_photons()
    params = PL.plate_params(scene, du0)
    px, py, flux = (t.float().cuda() for t in (ph[0], ph[1], ph[4]))
    Ep, xp, Mp, cp, radius = PL.refract_forward(h.cuda(), px, py, flux, params)
    rE, rx, rM, rc, rr = torch_inputs64(h, scene, ph)
    torch.cuda.synchronize()
    assert rel_l2(xp.cpu(), rx) < 1e-6
    assert rel_l2(Ep.cpu(), rE) < 1e-4
    assert rel_l2(Mp.cpu(), rM) < 1e-4
    assert rel_l2(radius.cpu(), rr) < 1e-4
    assert torch.equal(cp.cpu(), rc)


def test_refract_backward_matches_float64_autograd(cuda):
    from shapefromcaustics_b200 import plate as PL
    scene, h, ph, du0 = scene_and_photons(seed=3)
    params = PL.plate_params(scene, du0)
    n = ph[0].numel()
    g = torch.Generator().manual_seed(0)
    gE = torch.randn(n, generator=g, dtype=torch.float64)
    gX = torch.randn((2, n), generator=g, dtype=torch.float64)
    gM = torch.randn((2, 3, n), generator=g, dtype=torch.float64) * 1e-3
    gM[:, 2] = 0
    px, py, flux = (t.float().cuda() for t in (ph[0], ph[1], ph[4]))
    gh = PL.refract_backward(h.cuda(), px, py, flux, params, gE.float().cuda(), gX.float().cuda(),
                             gM.float().cuda())
    hd = h.double().requires_grad_(True)
    px64, py64, Du0, Dv0, flux64 = (t.double() for t in ph)
    Ep, xp, Mp, cp, radius = RF.receiver_splat_inputs(hd, scene, (px64, py64, Du0, Dv0, flux64))
    L = (Ep * gE).sum() + (xp * gX).sum() + (Mp * gM).sum()
    (ref,) = torch.autograd.grad(L, hd)
    torch.cuda.synchronize()
    assert rel_l2(gh.cpu(), ref) < 1e-3


def test_plate_splat_end_to_end_gradient(cuda):
    from shapefromcaustics_b200 import plate as PL
    scene, h, ph, du0 = scene_and_photons(seed=5)
    params = PL.plate_params(scene, du0)
    shape = (1, 128, 128)
    G = torch.randn(shape, generator=torch.Generator().manual_seed(1), dtype=torch.float64)
    px, py, flux = (t.float().cuda() for t in (ph[0], ph[1], ph[4]))
    for keep in (True, False):
        hv = h.cuda().requires_grad_(True)
        img = PL.PlateSplat.apply(hv, px, py, flux, params, shape, 20, keep)
        (img * G.float().cuda()).sum().backward()
        # FP64 reference: float64 chain, FP64 oracle splat and backward
        hd = h.double().requires_grad_(True)
        Ep, xp, Mp, cp, radius = RF.receiver_splat_inputs(
            hd, scene, tuple(t.double() for t in ph))
        a = [t.detach().numpy() for t in (Ep, xp, Mp, cp, radius)]
        rimg = O.forward(*a, shape, 20)
        gE, gX, gM = O.backward(G.numpy(), *a, 20)
        L = (Ep * torch.from_numpy(gE)).sum() + (xp * torch.from_numpy(gX)).sum() + \
            (Mp * torch.from_numpy(gM)).sum()
        (ref,) = torch.autograd.grad(L, hd)
        torch.cuda.synchronize()
        assert rel_l2(img.detach().cpu(), rimg) < 1e-4
        assert rel_l2(hv.grad.cpu(), ref) < 1e-3


@pytest.mark.parametrize("vol", ["low", "mid", "high"])
def test_landweber_update_matches_reference_ops(cuda, vol):
    from oracle.landweber_ref import landweber_update_reference
    from shapefromcaustics_b200.landweber import LandweberParams, landweber_update
    g = torch.Generator().manual_seed(3)
    H, W = 130, 97
    d = torch.rand((H, W), generator=g) * 0.2
    grad = torch.randn((H, W), generator=g)
    mask = (torch.rand((H, W), generator=g) > 0.3).float()
    s = float((mask * d).sum())
    d1, d2 = {"low": (2 * s, 3 * s), "mid": (0.5 * s, 3 * s), "high": (0.2 * s, 0.4 * s)}[vol]
    p = LandweberParams(tau=0.05, alpha=0.1, lower=0.0, upper=0.15, d1=d1, d2=d2, gamma=0.1,
                        radius=2)
    ref = landweber_update_reference(d.double(), grad.double(), mask.double(), p)
    out = landweber_update(d.cuda(), grad.cuda(), mask.cuda(), p)
    torch.cuda.synchronize()
    assert rel_l2(out.cpu(), ref) < 1e-5


def test_photon_source_matches_philox_restatement(cuda):
    """The device photon source reproduces the numpy Philox4x32-10 restatement bit for bit
    (odd photon count, nonzero counter offset, 64-bit seed), and successive calls advanced by
    the returned offset draw disjoint streams."""
    from oracle import philox as P
    from shapefromcaustics_b200.landweber import photon_source
    seed = 0x1234_5678_9ABC
    px, py, nxt = photon_source(5, 7, 3, 0.25, seed, 11, "cuda")
    torch.cuda.synchronize()
    rx, ry = P.photon_source(5, 7, 3, 0.25, seed, 11)
    assert nxt == 11 + 53
    assert np.array_equal(px.cpu().numpy(), rx) and np.array_equal(py.cpu().numpy(), ry)
    qx, qy, _ = photon_source(5, 7, 3, 0.25, seed, nxt, "cuda")
    sx, sy = P.photon_source(5, 7, 3, 0.25, seed, nxt)
    assert np.array_equal(qx.cpu().numpy(), sx)
    assert not np.array_equal(qx.cpu().numpy(), rx)
    # many photons: offsets uniform inside the texel
    px, py, _ = photon_source(64, 64, 16, 1.0, 7, 0, "cuda")
    t = torch.arange(px.numel(), device="cuda") % (64 * 64)
    jx = (px - ((t % 64).float() - 31.5)).cpu().numpy()
    assert abs(jx.mean()) < 5e-3 and abs(jx.var() - 1 / 12) < 2e-3
    assert jx.min() >= -0.5 and jx.max() <= 0.5  # (ix + j rounds to the texel edge at most)


def test_refract_forward_matches_the_reference_functions_fixture(cuda):
    """pds_refract_forward_f32 against the plate's chain composed from the reference's own
    functions in float64 (tests/golden/refraction_ref.npz; float32 kernel, float64 fixture)."""
    import os
    from shapefromcaustics_b200 import plate as PL
    gold = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                "refraction_ref.npz"))
    texel, ior, dist, half, du0 = (float(v) for v in gold["chain_params"])
    scene = RF.PlateScene(texel=texel, ior=ior, receiver_distance=dist, receiver_half=half,
                          light_dir=tuple(gold["chain_light"]))
    params = PL.plate_params(scene, du0)
    h = torch.from_numpy(gold["chain_h"]).float().cuda()
    px, py, flux = (torch.from_numpy(gold[k]).float().cuda()
                    for k in ("chain_px", "chain_py", "chain_flux"))
    Ep, xp, Mp, cp, radius = PL.refract_forward(h, px, py, flux, params)
    torch.cuda.synchronize()
    assert bool((cp >= 0).all())
    assert rel_l2(xp.cpu(), gold["chain_xp"]) < 1e-6
    assert rel_l2(Ep.cpu(), gold["chain_Ep"]) < 1e-4
    assert rel_l2(Mp.cpu(), gold["chain_Mp"]) < 1e-4
    assert rel_l2(radius.cpu(), gold["chain_radius"]) < 1e-4


def test_config2_gpu_gradient_matches_fp64_central_differences(cuda):
    """The 256^2 Landweber configuration in full on the GPU (float32 refraction + splat
    kernels, PlateSplat): the height-field gradient of 0.5 |I - T|^2 against FP64 central
    differences on 64 random texels (texels whose photons keep their truncation boxes under
    the steps)."""
    import plate_fd as PF
    from shapefromcaustics_b200 import plate as PL
    scene, h, t, photons, du0 = PF.config2()
    target = PF.splat64(t, scene, photons)
    params = PL.plate_params(scene, du0)
    px, py, _, _, flux = (x.float().cuda() for x in photons)
    shape = (1, PF.IMAGE, PF.IMAGE)
    hv = h.float().cuda().requires_grad_(True)
    img = PL.PlateSplat.apply(hv, px, py, flux, params, shape, PF.MPR, True)
    loss = 0.5 * ((img - torch.from_numpy(target).float().cuda()) ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    texels, skipped = PF.smooth_texels(h, scene, photons, 64)
    an = np.array([float(hv.grad[i, j]) for (i, j) in texels])
    fd, smooth = PF.fd_gradient(h, target, scene, photons, texels)
    assert smooth.all() and skipped < 64
    err = np.linalg.norm(fd - an) / np.linalg.norm(fd)
    assert err < 1e-3, (err, fd, an)


def test_point_light_source_matches_compute_point_light_dirs(cuda):
    """pds_point_light_source_f32 with the reference's own uniform numbers reproduces the
    reference's compute_point_light_dirs (tests/golden/refraction_ref.npz; float32 kernel,
    float64 fixture), and with its Philox numbers the FP64 restatement."""
    import os
    from oracle import point_light as PLR
    from shapefromcaustics_b200 import plate as PL
    gold = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                "refraction_ref.npz"))
    coords = gold["plight_coords"]
    z, _, sims, inner, smooth, energy = (float(v) for v in gold["plight_params"])
    rect = (coords[0].min(), coords[1].min(), coords[0].max(), coords[1].max())
    light = PL.point_light(gold["plight_light"], rect, z, smooth, energy, int(sims), int(inner))
    coeffs = torch.from_numpy(gold["plight_coeffs"].reshape(2, -1)).float().cuda()
    d, dt, dp, flux, _ = PL.point_light_source(light, coeffs.shape[1], "cuda", coeffs=coeffs)
    torch.cuda.synchronize()
    assert rel_l2(d.cpu().numpy().T, gold["plight_direction"]) < 1e-6
    assert rel_l2(dt.cpu().numpy().T, gold["plight_Dtheta"]) < 1e-5
    assert rel_l2(dp.cpu().numpy().T, gold["plight_Dphi"]) < 1e-5
    assert rel_l2(flux.cpu().numpy(), gold["plight_flux"]) < 1e-6
    # Philox numbers, three wavelengths per direction, against the restatement
    light3 = PL.point_light((0.3, -0.1, 12.0), (-2.0, -1.5, 2.0, 1.5), 1.0, 4.0, 1e-4, 16, 32, 3)
    n_dir = 5001
    d, dt, dp, flux, nxt = PL.point_light_source(light3, n_dir, "cuda", seed=77, offset=5)
    torch.cuda.synchronize()
    u0, u1 = PLR.philox_coeffs(n_dir, 77, 5)
    rd, rt, rp, rf = PLR.point_light((0.3, -0.1, 12.0), (-2.0, -1.5, 2.0, 1.5), 1.0, u0, u1, 4.0,
                                     1e-4, 16, 32, 3)
    assert nxt == 5 + (n_dir + 1) // 2 and d.shape == (3, 3 * n_dir)
    assert rel_l2(d.cpu().numpy().T, rd) < 1e-6
    assert rel_l2(dt.cpu().numpy().T, rt) < 1e-5
    assert rel_l2(flux.cpu().numpy(), rf) < 1e-6


def point_scene(n=48, n_dir=20000, seed=2):
    """A point light 40 mm above a 48 x 48 plate (texel 0.4 mm), photons from the device
    source, evaluated in float64 on their float32 values."""
    from shapefromcaustics_b200 import plate as PL
    scene = RF.PlateScene(texel=0.4, receiver_distance=30.0, receiver_half=12.0)
    h = RF.height_field_bumps(n, n, seed=seed, bumps=10, base=1.0, amp=(0.0, 0.05),
                              width=(2.0, 6.0)).float()
    half = 0.5 * (n - 1) * scene.texel
    rect = (-half + 0.2, -half + 0.2, half - 0.2, half - 0.2)
    light = PL.point_light((0.5, -0.4, 40.0), rect, 1.0, 3.0, 1.0, 1, 1, 1)
    d, dt, dp, flux, _ = PL.point_light_source(light, n_dir, "cuda", seed=seed)
    return scene, h, light, (d, dt, dp, flux)


def test_point_light_refract_forward_matches_float64_chain(cuda):
    from shapefromcaustics_b200 import plate as PL
    scene, h, light, (d, dt, dp, flux) = point_scene()
    params = PL.plate_params(scene, 0.0)
    Ep, xp, Mp, cp, radius = PL.refract_point_forward(h.cuda(), light, params, d, dt, dp, flux)
    torch.cuda.synchronize()
    pos = tuple(light.position)
    rE, rx, rM, rc, rr = RF.point_light_splat_inputs(
        h.double(), scene, pos, d.double().cpu(), dt.double().cpu(), dp.double().cpu(),
        flux.double().cpu(), float(light.plane_z))
    assert torch.equal(cp.cpu(), rc) and bool((rc >= 0).all())
    assert rel_l2(xp.cpu(), rx) < 1e-6
    assert rel_l2(Ep.cpu(), rE) < 1e-4
    assert rel_l2(Mp.cpu(), rM) < 1e-4
    assert rel_l2(radius.cpu(), rr) < 1e-4


def test_point_light_refract_backward_matches_float64_autograd(cuda):
    from shapefromcaustics_b200 import plate as PL
    scene, h, light, (d, dt, dp, flux) = point_scene(seed=3)
    params = PL.plate_params(scene, 0.0)
    n = flux.numel()
    g = torch.Generator().manual_seed(0)
    gE = torch.randn(n, generator=g, dtype=torch.float64)
    gX = torch.randn((2, n), generator=g, dtype=torch.float64)
    gM = torch.randn((2, 3, n), generator=g, dtype=torch.float64) * 1e-3
    gM[:, 2] = 0
    gh = PL.refract_point_backward(h.cuda(), light, params, d, dt, dp, flux, gE.float().cuda(),
                                   gX.float().cuda(), gM.float().cuda())
    hd = h.double().requires_grad_(True)
    Ep, xp, Mp, cp, radius = RF.point_light_splat_inputs(
        hd, scene, tuple(light.position), d.double().cpu(), dt.double().cpu(), dp.double().cpu(),
        flux.double().cpu(), float(light.plane_z))
    L = (Ep * gE).sum() + (xp * gX).sum() + (Mp * gM).sum()
    (ref,) = torch.autograd.grad(L, hd)
    torch.cuda.synchronize()
    assert rel_l2(gh.cpu(), ref) < 1e-3


def test_point_plate_splat_end_to_end_gradient(cuda):
    from shapefromcaustics_b200 import plate as PL
    scene, h, light, (d, dt, dp, flux) = point_scene(seed=5)
    params = PL.plate_params(scene, 0.0)
    shape = (1, 128, 128)
    G = torch.randn(shape, generator=torch.Generator().manual_seed(1), dtype=torch.float64)
    hv = h.cuda().requires_grad_(True)
    img = PL.PointPlateSplat.apply(hv, d, dt, dp, flux, light, params, shape, 20)
    (img * G.float().cuda()).sum().backward()
    hd = h.double().requires_grad_(True)
    Ep, xp, Mp, cp, radius = RF.point_light_splat_inputs(
        hd, scene, tuple(light.position), d.double().cpu(), dt.double().cpu(), dp.double().cpu(),
        flux.double().cpu(), float(light.plane_z))
    a = [t.detach().numpy() for t in (Ep, xp, Mp, cp, radius)]
    rimg = O.forward(*a, shape, 20)
    gE, gX, gM = O.backward(G.numpy(), *a, 20)
    L = (Ep * torch.from_numpy(gE)).sum() + (xp * torch.from_numpy(gX)).sum() + \
        (Mp * torch.from_numpy(gM)).sum()
    (ref,) = torch.autograd.grad(L, hd)
    torch.cuda.synchronize()
    assert rel_l2(img.detach().cpu(), rimg) < 1e-4
    assert rel_l2(hv.grad.cpu(), ref) < 1e-3


def plate_batch(n_field=48, seed=7):
    """Five simulations of one plate, each with its own tilt, wavelength, photon count and
    image size."""
    from shapefromcaustics_b200 import plate as PL
    from shapefromcaustics_b200.landweber import photon_source
    from shapefromcaustics_b200.scene import fused_silica
    rng = np.random.default_rng(seed)
    scene = RF.PlateScene(texel=0.4, receiver_distance=30.0, receiver_half=14.0)
    h = RF.height_field_bumps(n_field, n_field, seed=seed, bumps=10, base=1.0,
                              amp=(0.0, 0.05), width=(2.0, 8.0)).float().cuda()
    sims, photons = [], []
    offset = 0
    for k, (per, img) in enumerate([(2, 64), (1, 128), (4, 96), (3, 64), (1, 256)]):
        th, ph = np.radians(5.0) * rng.random(), 2 * np.pi * rng.random()
        light = (np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), -np.cos(th))
        s = RF.PlateScene(texel=0.4, ior=float(fused_silica(0.45 + 0.2 * rng.random())),
                          receiver_distance=30.0, receiver_half=14.0, light_dir=light)
        p = PL.plate_params(s, 3.0 * 2.0 * s.receiver_half / img)
        px, py, offset = photon_source(n_field, n_field, per, s.texel, 11, offset, "cuda")
        n = px.numel()
        sims.append((n, (1, img, img), p))
        photons.append((px, py, torch.full((n,), 1.0 / n, device="cuda")))
    return h, sims, photons


def test_batched_plate_equals_the_per_simulation_plates(cuda):
    from shapefromcaustics_b200 import plate as PL
    h, sims, photons = plate_batch()
    batch = PL.BatchedPlate(sims, 20, "cuda")
    cat = [torch.cat([p[k] for p in photons]).contiguous() for k in range(3)]
    hv = h.clone().requires_grad_(True)
    flat = PL.BatchedPlateSplat.apply(hv, *cat, batch)
    g = torch.randn(flat.shape, generator=torch.Generator("cuda").manual_seed(3), device="cuda")
    (flat * g).sum().backward()
    imgs = batch.images(flat.detach())
    gsum = torch.zeros_like(h)
    off = 0
    for (n, shape, p), (px, py, flux), img in zip(sims, photons, imgs):
        hs = h.clone().requires_grad_(True)
        ref = PL.PlateSplat.apply(hs, px, py, flux, p, shape, 20, True)
        gs = g[off:off + ref.numel()].view(shape)
        (ref * gs).sum().backward()
        gsum += hs.grad
        off += ref.numel()
        assert rel_l2(img.cpu(), ref.detach().cpu()) < 1e-5
    torch.cuda.synchronize()
    assert rel_l2(hv.grad.cpu(), gsum.cpu()) < 1e-5


def test_batched_plate_kept_and_recomputed_inputs_agree(cuda):
    """The backward on the forward's kept splat inputs and on inputs recomputed from the
    height field give the same height gradient (same kernels on the same inputs; only the
    order of the float atomic sums into the field differs)."""
    from shapefromcaustics_b200 import plate as PL
    h, sims, photons = plate_batch()
    cat = [torch.cat([p[k] for p in photons]).contiguous() for k in range(3)]
    grads = []
    for keep in (True, False):
        batch = PL.BatchedPlate(sims, 20, "cuda", keep_inputs=keep)
        img = batch.forward(h, *cat)
        g = torch.randn(img.shape, generator=torch.Generator("cuda").manual_seed(4),
                        device="cuda")
        grads.append(batch.backward(h, *cat, g))
        assert (batch.splat.inputs is not None) == keep
    torch.cuda.synchronize()
    assert rel_l2(grads[0].cpu(), grads[1].cpu()) < 1e-6


def test_refraction_backward_from_gradient_records_equals_arrays(cuda):
    """The refraction backward reading the splat gradients from the plan's gradient records
    (``records=True`` + ``pds_refract_backward_planned_f32``, the batch variant likewise)
    gives the height gradient of the spread arrays' path (same values; only the order of the
    float atomic sums into the field differs)."""
    from shapefromcaustics_b200 import plate as PL
    from shapefromcaustics_b200._lib import check, lib
    from shapefromcaustics_b200.splatting import SplatPlan, _ptr, _stream
    scene, h, ph, du0 = scene_and_photons(seed=9)
    params = PL.plate_params(scene, du0)
    h = h.cuda()
    px, py, flux = (t.float().cuda() for t in (ph[0], ph[1], ph[4]))
    shape = (1, 96, 96)
    plan = SplatPlan(*PL.refract_forward(h, px, py, flux, params), shape, 20)
    g = torch.randn(shape, generator=torch.Generator("cuda").manual_seed(5), device="cuda")
    plan.forward()
    gE, gX, gM = plan.backward(g)
    gh_arrays = PL.refract_backward(h, px, py, flux, params, gE, gX, gM)
    assert plan.backward(g, records=True) is None
    gh_records = PL.refract_backward_planned(h, px, py, flux, params, plan)
    torch.cuda.synchronize()
    assert float(gh_arrays.abs().max()) > 0
    assert rel_l2(gh_records.cpu(), gh_arrays.cpu()) < 1e-6
    # a batch of plates: BatchedPlate.backward (records) against the arrays' path
    hb, sims, photons = plate_batch()
    cat = [torch.cat([p[k] for p in photons]).contiguous() for k in range(3)]
    batch = PL.BatchedPlate(sims, 20, "cuda")
    img = batch.forward(hb, *cat)
    gb = torch.randn(img.shape, generator=torch.Generator("cuda").manual_seed(6), device="cuda")
    gh_b_records = batch.backward(hb, *cat, gb)
    gE, gX, gM = batch.splat.backward(gb)
    gh_b_arrays = torch.zeros_like(hb)
    with torch.cuda.device(hb.device):
        check(lib().pds_batch_refract_backward_f32(
            _ptr(hb), hb.shape[0], hb.shape[1], _ptr(batch.plates_dev), _ptr(batch.begins_dev),
            batch.n_sims, _ptr(cat[0]), _ptr(cat[1]), _ptr(cat[2]), batch.n_total, _ptr(gE),
            _ptr(gX), _ptr(gM), _ptr(gh_b_arrays), _stream(hb.device)))
    torch.cuda.synchronize()
    assert float(gh_b_arrays.abs().max()) > 0
    assert rel_l2(gh_b_records.cpu(), gh_b_arrays.cpu()) < 1e-6


def test_landweber_iteration_replays_from_a_cuda_graph(cuda):
    """The autograd Landweber iteration (refraction + splat forward, data term, backward
    through both, fused update) captured once in a CUDA graph: each replay gives the eager
    iteration's update (the forward's sums are reassociated by the plan's photon order, so
    to within float rounding, not bit for bit)."""
    from shapefromcaustics_b200 import plate as PL
    from shapefromcaustics_b200.landweber import LandweberParams, landweber_update
    scene, h, ph, du0 = scene_and_photons(seed=11)
    params = PL.plate_params(scene, du0)
    dev = torch.device("cuda")
    px, py, flux = (t.float().to(dev) for t in (ph[0], ph[1], ph[4]))
    shape = (1, 128, 128)
    with torch.no_grad():
        target = PL.PlateSplat.apply(h.to(dev) * 1.02, px, py, flux, params, shape, 20, False)
    base = 1.0
    d0 = (h.to(dev) - base).contiguous()
    d = d0.clone()
    mask = torch.ones_like(d)
    vol = float(d0.sum())
    lp = LandweberParams(tau=1e-2, d1=0.75 * vol, d2=1.25 * vol)
    ws = torch.empty(1 << 20, dtype=torch.uint8, device=dev)

    def step():
        d.copy_(d0)
        hv = (base + d).requires_grad_(True)
        img = PL.PlateSplat.apply(hv, px, py, flux, params, shape, 20, True)
        (0.5 * ((img - target) ** 2).sum()).backward()
        landweber_update(d, hv.grad, mask, lp, ws)

    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(3):
            step()
    torch.cuda.synchronize()
    eager = d.clone()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        step()
    for _ in range(2):
        d.zero_()
        graph.replay()
        torch.cuda.synchronize()
        upd = (eager - d0).norm()
        assert float(upd) > 0
        assert float((d - eager).norm() / upd) < 1e-4
    del graph


def test_refract_backward_independent_of_photon_order(cuda):
    """The refraction backward sums a CTA's patches in a shared region when its photons' cells
    are compact (raster order) and adds them with global atomics when they are scattered; both
    paths, and regions that alternate between consecutive blocks, give the same field gradient
    (to within the float reassociation of the sums). 262 144 photons give each CTA of the
    three-a-SM grid two or three blocks of 256."""
    from shapefromcaustics_b200 import plate as PL
    scene, h, ph, du0 = scene_and_photons(n=256, seed=13)
    params = PL.plate_params(scene, du0)
    n = ph[0].numel()
    g = torch.Generator().manual_seed(5)
    gE = torch.randn(n, generator=g)
    gX = torch.randn((2, n), generator=g)
    gM = torch.randn((2, 3, n), generator=g) * 1e-3
    gM[:, 2] = 0
    px, py, flux = (t.float() for t in (ph[0], ph[1], ph[4]))
    dev = torch.device("cuda")
    hd = h.to(dev)
    ordered = PL.refract_backward(hd, px.to(dev), py.to(dev), flux.to(dev), params, gE.to(dev),
                                  gX.to(dev), gM.to(dev))
    perm = torch.randperm(n, generator=g)
    shuffled = PL.refract_backward(hd, px[perm].to(dev), py[perm].to(dev), flux[perm].to(dev),
                                   params, gE[perm].to(dev), gX[:, perm].contiguous().to(dev),
                                   gM[:, :, perm].contiguous().to(dev))
    torch.cuda.synchronize()
    assert n > 2 * 256 * 148 * 3
    assert float(ordered.norm()) > 0
    assert rel_l2(shuffled.cpu(), ordered.cpu()) < 1e-5
