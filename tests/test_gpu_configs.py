"""Parity of the CUDA path with the FP64 oracle on the benchmark configurations at their
stated sizes (not scaled-down analogues).

  - the CPU-runnable configuration in full: 2^20 photons, 512^2, seed 0, half uniform and half
    in 8 Gaussian clusters (sigma 20 px), s ~ logU[0.5, 4] px;
  - the 64-simulation uneven batch that ``bench.py`` times (its rank-0 seed): its first 16
    simulations (13.4 M photons, every image size 256^2, 512^2 and 1024^2 among them) through
    one batched plan, forward and backward;
  - the contention configuration's generator on 2048^2 (80 % of the photons on 4 caustic
    curves of 1.5 px cross-section, s ~ logU[0.25, 16] px), subsampled to 2^22 photons so the
    oracle finishes in seconds.

Tolerances (written in the target): forward images relative L2 <= 1e-5, gradients relative
L2 <= 1e-4, against the FP64 oracle on the same float32 inputs.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from shapefromcaustics_b200 import synthetic as S

pytestmark = pytest.mark.gpu

FWD_TOL = 1e-5
GRAD_TOL = 1e-4
MPR = 20


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def oracle(ph, shape, grad):
    npy = [t.detach().cpu().numpy() for t in ph]
    img = O.forward(*npy, shape, MPR)
    g = O.backward(grad.detach().cpu().numpy().astype(np.float64), *npy, MPR)
    return img, g


def check(img, grads, rimg, rgrads):
    errs = {"image": rel_l2(img, rimg)}
    for k, a, b in zip(("grad_Ep", "grad_xp", "grad_Mp"), grads, rgrads):
        errs[k] = rel_l2(a, b)
    bad = {k: v for k, v in errs.items() if not v <= (FWD_TOL if k == "image" else GRAD_TOL)}
    assert not bad, errs
    return errs


def test_cpu_runnable_configuration_in_full(cuda):
    from shapefromcaustics_b200 import pds_backward, pds_forward
    shape = (1, 512, 512)
    ph = S.uniform_cluster_photons(2 ** 20, 512, 512, seed=0)
    G = S.upstream_grad(shape, seed=1)
    dev = [t.cuda() for t in ph]
    img = pds_forward(*dev, list(shape), MPR)[0]
    grads = pds_backward(G.cuda(), *dev, MPR)
    torch.cuda.synchronize()
    rimg, rg = oracle(ph, shape, G)
    check(img.cpu().numpy(), [g.cpu().numpy() for g in grads], rimg, rg)
    assert np.all(grads[2].cpu().numpy()[:, 2] == 0)


def test_benchmark_batch_first_16_simulations(cuda):
    from shapefromcaustics_b200.splatting import BatchedSplat
    seed = 1000  # bench.py's rank-0 batch
    specs = S.batch_specs(64, seed=seed)[:16]
    assert {H for _, (_, H, _) in specs} == {256, 512, 1024}
    photons = S.batch_photons(specs, seed=seed, device="cuda")
    grads = [S.upstream_grad(shape, seed=seed * 7919 + s, device="cuda").reshape(-1)
             for s, (_, shape) in enumerate(specs)]
    gflat = torch.cat(grads).contiguous()
    b = BatchedSplat(specs, MPR, "cuda:0")
    b.plan(*photons)
    flat = b.forward()
    gE, gX, gM = b.backward(gflat)
    torch.cuda.synchronize()
    imgs = b.images(flat)
    off = 0
    for s, (n, shape) in enumerate(specs):
        sl = slice(off, off + n)
        ph = (photons[0][sl], photons[1][:, sl], photons[2][:, :, sl], photons[3][:, sl],
              photons[4][sl])
        rimg, rg = oracle(ph, shape, grads[s].view(shape))
        check(imgs[s].cpu().numpy(), [gE[sl].cpu().numpy(), gX[:, sl].cpu().numpy(),
                                      gM[:, :, sl].cpu().numpy()], rimg, rg)
        off += n


def test_contention_configuration_on_2048(cuda):
    from shapefromcaustics_b200 import pds_backward, pds_forward
    shape = (1, 2048, 2048)
    ph = S.caustic_curve_photons(2 ** 22, 2048, 2048, seed=0, device="cuda")
    G = S.upstream_grad(shape, seed=2, device="cuda")
    img = pds_forward(*ph, list(shape), MPR)[0]
    grads = pds_backward(G, *ph, MPR)
    torch.cuda.synchronize()
    rimg, rg = oracle(ph, shape, G)
    check(img.cpu().numpy(), [g.cpu().numpy() for g in grads], rimg, rg)
