"""Parity of the sm_100a splatting kernels (through the C ABI) with the FP64 oracle.

Tolerances (stated by the target): forward images relative L2 <= 1e-5, gradients relative
L2 <= 1e-4, both against the FP64 oracle on the same float32 inputs.
"""
import ctypes

import numpy as np
import pytest
import torch

from oracle import oracle as O
from shapefromcaustics_b200 import synthetic as S

pytestmark = pytest.mark.gpu

FWD_TOL = 1e-5
GRAD_TOL = 1e-4


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def to_np(ts):
    return [t.detach().cpu().numpy() for t in ts]


def run_gpu(photons, shape, mpr, grad, cfg=None, dev="cuda:0"):
    from shapefromcaustics_b200 import splatting as SP
    E, X, M, C, R = (t.to(dev) for t in photons)
    if cfg is not None:
        SP.set_default_config(**cfg)
    try:
        img = SP.pds_forward(E, X, M, C, R, list(shape), mpr)[0]
        g = SP.pds_backward(grad.to(dev).contiguous(), E, X, M, C, R, mpr)
    finally:
        SP.set_default_config()
    torch.cuda.synchronize()
    return img.cpu().numpy(), to_np(g)


def run_oracle(photons, shape, mpr, grad):
    E, X, M, C, R = to_np(photons)
    img = O.forward(E, X, M, C, R, shape, mpr)
    g = O.backward(grad.numpy().astype(np.float64), E, X, M, C, R, mpr)
    return img, g


def assert_parity(photons, shape, mpr, grad=None, cfg=None, fwd_tol=FWD_TOL, grad_tol=GRAD_TOL):
    if grad is None:
        grad = S.upstream_grad(shape, seed=7)
    img, (gE, gX, gM) = run_gpu(photons, shape, mpr, grad, cfg)
    rimg, (rE, rX, rM) = run_oracle(photons, shape, mpr, grad)
    assert rel_l2(img, rimg) <= fwd_tol, rel_l2(img, rimg)
    assert rel_l2(gE, rE) <= grad_tol, rel_l2(gE, rE)
    assert rel_l2(gX, rX) <= grad_tol, rel_l2(gX, rX)
    assert rel_l2(gM, rM) <= grad_tol, rel_l2(gM, rM)
    assert np.all(gM[:, 2] == 0)
    return img, rimg


def test_uniform_cluster_512(cuda):
    ph = S.uniform_cluster_photons(2 ** 17, 512, 512, seed=0)
    assert_parity(ph, (1, 512, 512), 20)


@pytest.mark.parametrize("cfg", [dict(tile=16), dict(tile=32), dict(chunk=256),
                                 dict(class_bits=-1), dict(class_bits=4, chunk=4096),
                                 dict(tile=32, apron_max=3), dict(walk=2),
                                 dict(walk=2, tile=16, class_bits=1), dict(min_blocks=2),
                                 dict(coop_radius=1), dict(coop_radius=-1),
                                 dict(coop_radius=2, min_blocks=2), dict(walk=1),
                                 dict(walk=1, coop_radius=5), dict(walk=3, coop_radius=4, tile=32),
                                 dict(min_blocks=4), dict(min_blocks=4, class_bits=3),
                                 dict(walk=3, class_bits=5), dict(walk=4, min_blocks=2),
                                 dict(walk=4, class_bits=5), dict(walk=4, tile=32),
                                 dict(walk=4, coop_radius=4), dict(walk=4, class_bits=-1),
                                 dict(walk=4, tile=16, apron_max=5), dict(min_blocks=3)])
def test_tuning_variants(cuda, cfg):
    ph = S.uniform_cluster_photons(2 ** 15, 256, 256, seed=1)
    assert_parity(ph, (1, 256, 256), 20, cfg=cfg)


def test_non_square_ragged_image_and_channels(cuda):
    n = 20000
    E, X, M, C, R = S.uniform_cluster_photons(n, 70, 100, seed=2, s_range=(0.5, 6.0))
    g = torch.Generator().manual_seed(5)
    C = torch.randint(-1, 4, (1, n), generator=g)  # channels -1..3 with C = 3: some skipped
    assert_parity((E, X, M, C, R), (3, 70, 100), 20)


def test_wide_footprints_take_the_direct_path(cuda):
    # radii up to 40 px > apron_max (8): direct path; mpr 30 truncates some boxes
    ph = S.uniform_cluster_photons(3000, 128, 128, seed=3, s_range=(0.5, 40.0))
    assert_parity(ph, (1, 128, 128), 30, cfg=dict(apron_max=8))


@pytest.mark.parametrize("cfg", [dict(walk=1, coop_radius=3), dict(walk=1, coop_radius=-1),
                                 dict(), dict(class_bits=4), dict(walk=2), dict(walk=3),
                                 dict(walk=4, min_blocks=2)])
def test_caustic_curves_large_footprints(cuda, cfg):
    # the contention workload's shape at a small size: most photons on thin curves
    ph = S.caustic_curve_photons(2 ** 16, 256, 256, seed=13, s_range=(0.25, 16.0))
    assert_parity(ph, (1, 256, 256), 20, cfg=cfg)


def test_photons_partly_and_fully_off_image(cuda):
    n = 8000
    g = torch.Generator().manual_seed(4)
    pos = torch.rand((2, n), generator=g, dtype=torch.float64) * 80 - 8  # [-8, 72) on 64^2
    th = torch.rand(n, generator=g, dtype=torch.float64) * np.pi
    s1 = 0.5 + torch.rand(n, generator=g, dtype=torch.float64) * 5
    s2 = 0.5 + torch.rand(n, generator=g, dtype=torch.float64) * 5
    e = torch.rand(n, generator=g, dtype=torch.float64) - 0.2  # some E <= 0
    ph = S.photons_from_pixels(pos, th, s1, s2, e, 64, 64)
    assert_parity(ph, (1, 64, 64), 20)


def test_tiny_image_ellipse_quirk(cuda):
    ph = S.uniform_cluster_photons(500, 8, 8, seed=5, s_range=(2.0, 20.0), sigma=2.0)
    assert_parity(ph, (1, 8, 8), 20)


@pytest.mark.parametrize("mpr", [0, 1, -1])
def test_small_and_negative_max_pixel_radius(cuda, mpr):
    ph = S.uniform_cluster_photons(4000, 64, 64, seed=6)
    assert_parity(ph, (1, 64, 64), mpr)


@pytest.mark.parametrize("n", [0, 1, 255, 257])
def test_tiny_photon_counts(cuda, n):
    ph = S.uniform_cluster_photons(max(n, 1), 64, 64, seed=8)
    ph = tuple(t[..., :n].contiguous() for t in ph)
    img, rimg = assert_parity(ph, (1, 64, 64), 20)
    if n == 0:
        assert not img.any()


def test_dense_contention_hot_tile(cuda):
    # all photons in a 6x6 px spot: one tile segment spans many chunks
    n = 200000
    g = torch.Generator().manual_seed(9)
    pos = 100.0 + torch.randn((2, n), generator=g, dtype=torch.float64) * 1.5
    th = torch.rand(n, generator=g, dtype=torch.float64) * np.pi
    s = torch.exp(torch.rand((2, n), generator=g, dtype=torch.float64) * np.log(64) + np.log(0.25))
    e = 0.5 + torch.rand(n, generator=g, dtype=torch.float64) * 0.5
    ph = S.photons_from_pixels(pos, th, s[0], s[1], e, 256, 256)
    assert_parity(ph, (1, 256, 256), 20)


def test_planned_and_unplanned_agree_bitwise_in_backward(cuda):
    from shapefromcaustics_b200.splatting import SplatPlan, pds_backward
    E, X, M, C, R = (t.cuda() for t in S.uniform_cluster_photons(50000, 256, 256, seed=10))
    G = S.upstream_grad((1, 256, 256), seed=3).cuda()
    plan = SplatPlan(E, X, M, C, R, (1, 256, 256), 20)
    a = plan.backward(G)
    b = pds_backward(G, E, X, M, C, R, 20)
    for u, v in zip(a, b):
        assert torch.equal(u, v)


def test_autograd_function_and_shim(cuda):
    import shapefromcaustics_b200 as P
    mod = P.shim.install()
    import PhotonDifferentialSplatting as PDSmod
    assert PDSmod.pds_forward is P.pds_forward
    E, X, M, C, R = (t.cuda() for t in S.uniform_cluster_photons(30000, 128, 128, seed=11))
    E.requires_grad_(True); X.requires_grad_(True); M.requires_grad_(True)
    G = S.upstream_grad((1, 128, 128), seed=4).cuda()
    img = P.PDS.apply(E, X, M, C, R, (1, 128, 128), 20)
    (img * G).sum().backward()
    rimg, (rE, rX, rM) = run_oracle((E.detach().cpu(), X.detach().cpu(), M.detach().cpu(),
                                     C.cpu(), R.cpu()), (1, 128, 128), 20, G.cpu())
    assert rel_l2(img.detach().cpu().numpy(), rimg) <= FWD_TOL
    assert rel_l2(E.grad.cpu().numpy(), rE) <= GRAD_TOL
    assert rel_l2(X.grad.cpu().numpy(), rX) <= GRAD_TOL
    assert rel_l2(M.grad.cpu().numpy(), rM) <= GRAD_TOL
    # the same with the plan rebuilt in backward
    P.set_keep_plan(False)
    try:
        E.grad = None
        img2 = P.PDS.apply(E, X, M, C, R, (1, 128, 128), 20)
        (img2 * G).sum().backward()
        assert rel_l2(E.grad.cpu().numpy(), rE) <= GRAD_TOL
    finally:
        P.set_keep_plan(True)


def test_input_validation_messages(cuda):
    from shapefromcaustics_b200 import pds_forward
    E, X, M, C, R = (t.cuda() for t in S.uniform_cluster_photons(100, 32, 32, seed=12))
    with pytest.raises(RuntimeError, match="must be a CUDA tensor"):
        pds_forward(E.cpu(), X, M, C, R, [1, 32, 32], 20)
    with pytest.raises(RuntimeError, match="must be contiguous"):
        pds_forward(E, X.t().contiguous().t(), M, C, R, [1, 32, 32], 20)
    with pytest.raises(RuntimeError, match="don't match"):
        pds_forward(E[:50].contiguous(), X, M, C, R, [1, 32, 32], 20)
    with pytest.raises(RuntimeError, match="2x3"):
        pds_forward(E, X, M[:, :2].contiguous(), C, R, [1, 32, 32], 20)
    with pytest.raises(RuntimeError, match="Long"):
        pds_forward(E, X, M, C.int(), R, [1, 32, 32], 20)
    with pytest.raises(RuntimeError, match="float32"):
        pds_forward(E.double(), X, M, C, R, [1, 32, 32], 20)


def test_batched_uneven_simulations_match_per_simulation_oracle(cuda):
    from shapefromcaustics_b200.splatting import BatchedSplat
    specs = [(3000, (1, 64, 64)), (0, (1, 32, 32)), (12000, (2, 96, 80)), (700, (1, 16, 16)),
             (40000, (1, 256, 256))]
    parts = []
    for s, (n, (C, H, W)) in enumerate(specs):
        ph = S.uniform_cluster_photons(max(n, 1), H, W, seed=100 + s, sigma=H / 8)
        ph = tuple(t[..., :n] for t in ph)
        if C > 1:
            ph = (ph[0], ph[1], ph[2], torch.randint(0, C, (1, n), generator=torch.Generator().manual_seed(s)), ph[4])
        parts.append(ph)
    cat = [torch.cat([p[k] for p in parts], dim=-1).contiguous().cuda() for k in range(5)]
    b = BatchedSplat(specs, 20, "cuda:0")
    b.plan(*cat)
    flat = b.forward()
    grads = [S.upstream_grad(shape, seed=50 + s) for s, (_, shape) in enumerate(specs)]
    gflat = torch.cat([g.reshape(-1) for g in grads]).cuda()
    gE, gX, gM = b.backward(gflat)
    torch.cuda.synchronize()
    imgs = b.images(flat)
    off = 0
    for s, ((n, shape), ph) in enumerate(zip(specs, parts)):
        rimg, (rE, rX, rM) = run_oracle(ph, shape, 20, grads[s])
        assert rel_l2(imgs[s].cpu().numpy(), rimg) <= FWD_TOL
        sl = slice(off, off + n)
        if n:
            assert rel_l2(gE[sl].cpu().numpy(), rE) <= GRAD_TOL
            assert rel_l2(gX[:, sl].cpu().numpy(), rX) <= GRAD_TOL
            assert rel_l2(gM[:, :, sl].cpu().numpy(), rM) <= GRAD_TOL
        off += n


@pytest.mark.parametrize("cfg", [None, dict(tile=32)])
def test_bucket_window_overflow_on_2048_images(cuda, cfg):
    # 2048^2 images: 32768 buckets a simulation at tile 64 (the plan's whole shared window) and
    # 131072 at tile 32, so CTAs that straddle the two simulations, or whose photons reach past
    # the window inside one, count and place those photons with global atomics
    from shapefromcaustics_b200 import _lib
    from shapefromcaustics_b200.splatting import BatchedSplat
    specs = [(2 ** 18 + 3001, (1, 2048, 2048)), (2 ** 17, (1, 2048, 2048))]
    parts = [S.uniform_cluster_photons(n, 2048, 2048, seed=300 + s) for s, (n, _) in
             enumerate(specs)]
    cat = [torch.cat([p[k] for p in parts], dim=-1).contiguous().cuda() for k in range(5)]
    b = BatchedSplat(specs, 20, "cuda:0", config=_lib.config(**(cfg or {})))
    b.plan(*cat)
    flat = b.forward()
    grads = [S.upstream_grad(shape, seed=60 + s) for s, (_, shape) in enumerate(specs)]
    gflat = torch.cat([g.reshape(-1) for g in grads]).cuda()
    gE, gX, gM = b.backward(gflat)
    torch.cuda.synchronize()
    imgs = b.images(flat)
    off = 0
    for s, ((n, shape), ph) in enumerate(zip(specs, parts)):
        rimg, (rE, rX, rM) = run_oracle(ph, shape, 20, grads[s])
        assert rel_l2(imgs[s].cpu().numpy(), rimg) <= FWD_TOL
        sl = slice(off, off + n)
        assert rel_l2(gE[sl].cpu().numpy(), rE) <= GRAD_TOL
        assert rel_l2(gX[:, sl].cpu().numpy(), rX) <= GRAD_TOL
        assert rel_l2(gM[:, :, sl].cpu().numpy(), rM) <= GRAD_TOL
        off += n


def test_simulations_sharing_an_image_are_summed(cuda):
    # the reference's caller sums its simulations' images (shape_from_caustics.py:351-353)
    from shapefromcaustics_b200 import _lib
    from shapefromcaustics_b200.splatting import BatchedSplat
    specs = [(5000, (1, 96, 96)), (7000, (1, 96, 96)), (3000, (1, 96, 96))]
    parts = [S.uniform_cluster_photons(n, 96, 96, seed=200 + s) for s, (n, _) in enumerate(specs)]
    cat = [torch.cat([p[k] for p in parts], dim=-1).contiguous().cuda() for k in range(5)]
    b = BatchedSplat(specs, 20, "cuda:0")
    # point every simulation at image 0
    t = (_lib.PdsSim * 3).from_buffer_copy(bytes(b.table_dev.cpu().numpy()))
    for k in range(3):
        t[k].image_offset = 0
    b.table_dev = torch.frombuffer(bytearray(bytes(t)), dtype=torch.uint8).cuda()
    b.image_elems = 96 * 96
    b.plan(*cat)
    img = b.forward()
    G = S.upstream_grad((1, 96, 96), seed=9)
    gE, gX, gM = b.backward(G.reshape(-1).cuda())
    torch.cuda.synchronize()
    allp = [torch.cat([p[k] for p in parts], dim=-1) for k in range(5)]
    rimg, (rE, rX, rM) = run_oracle(allp, (1, 96, 96), 20, G)
    assert rel_l2(img.view(1, 96, 96).cpu().numpy(), rimg) <= FWD_TOL
    assert rel_l2(gE.cpu().numpy(), rE) <= GRAD_TOL
    assert rel_l2(gX.cpu().numpy(), rX) <= GRAD_TOL
    assert rel_l2(gM.cpu().numpy(), rM) <= GRAD_TOL


def test_batched_graph_replay_equals_eager(cuda):
    from shapefromcaustics_b200.splatting import BatchedSplat
    specs = S.batch_specs(6, seed=3, n_range=(2 ** 10, 2 ** 14), sizes=(64, 128))
    photons = [t.cuda() for t in S.batch_photons(specs, seed=3)]
    b = BatchedSplat(specs, 20, "cuda:0")
    gflat = torch.randn(b.image_elems, device="cuda", generator=torch.Generator("cuda").manual_seed(0))
    b.plan(*photons)
    ref_img = b.forward().clone()
    ref_g = [t.clone() for t in b.backward(gflat)]
    out = torch.empty(b.image_elems, device="cuda")
    grads = tuple(torch.empty_like(t) for t in photons[:3])
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        b.plan(*photons); b.forward(out); b.backward(gflat, grads)
    torch.cuda.current_stream().wait_stream(s)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        b.plan(*photons)
        b.forward(out)
        b.backward(gflat, grads)
    out.zero_()
    graph.replay()
    torch.cuda.synchronize()
    assert rel_l2(out.cpu().numpy(), ref_img.cpu().numpy()) <= 1e-6
    for u, v in zip(grads, ref_g):
        assert torch.equal(u, v)


def test_autotuner_picks_and_caches_a_candidate(cuda):
    from shapefromcaustics_b200 import autotune
    specs = S.batch_specs(4, seed=5, n_range=(2 ** 10, 2 ** 13), sizes=(64, 128))
    photons = [t.cuda() for t in S.batch_photons(specs, seed=5)]
    gflat = torch.cat([S.upstream_grad(shape, seed=s).reshape(-1)
                       for s, (_, shape) in enumerate(specs)]).cuda()
    cands = [dict(tile=64, class_bits=5), dict(tile=32, class_bits=3, walk=1)]
    best, times = autotune.tune_batch(specs, photons, gflat, 20, torch.device("cuda"),
                                      candidates=cands, reps=1)
    assert best in cands and len(times) == 2 and all(t > 0 for t in times.values())
    assert autotune.cached(specs, 20) == best


def test_largest_apron_with_the_forward_record_staging(cuda):
    # max_pixel_radius 40: the 32-pixel apron, a 129 x 129 shared accumulator plus the
    # forward's two record staging buffers (82.9 KB a CTA), footprints up to the radius cap
    ph = S.caustic_curve_photons(2 ** 15, 384, 384, seed=21, s_range=(0.5, 40.0))
    assert_parity(ph, (1, 384, 384), 40)
