"""The photon-sharded path of one simulation through the CUDA splat ops, on one GPU.

Two ranks' shards of one simulation are run one after the other through
``sharded.sharded_forward`` / ``sharded.sharded_backward`` with the default (CUDA) ops and no
process group: the sum of the two partial images is the whole simulation's image, and each
shard's gradients are the whole simulation's gradients of its photons, both against the FP64
oracle (forward relative L2 <= 1e-5, gradients <= 1e-4).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from shapefromcaustics_b200 import sharded as SH
from shapefromcaustics_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("world", [2, 3])
def test_shards_through_the_cuda_ops_sum_to_the_simulation(cuda, world):
    shape = (1, 192, 160)
    n = 60001
    ph = S.uniform_cluster_photons(n, 192, 160, seed=31, sigma=12.0)
    dev_ph = [t.cuda() for t in ph]
    G = S.upstream_grad(shape, seed=6)
    total = torch.zeros(shape, device="cuda")
    grads = []
    for rank in range(world):
        local = SH.shard_photons(*dev_ph, rank, world)
        assert all(t.is_contiguous() for t in local)
        total += SH.sharded_forward(*local, list(shape), 20)[0]
        grads.append(SH.sharded_backward(G.cuda(), *local, 20))
    torch.cuda.synchronize()
    npy = [t.numpy() for t in ph]
    rimg = O.forward(*npy, shape, 20)
    rE, rX, rM = O.backward(G.numpy().astype(np.float64), *npy, 20)
    assert rel_l2(total.cpu().numpy(), rimg) <= 1e-5
    for rank, (gE, gX, gM) in enumerate(grads):
        b, e = SH.shard_range(n, rank, world)
        assert rel_l2(gE.cpu().numpy(), rE[b:e]) <= 1e-4
        assert rel_l2(gX.cpu().numpy(), rX[:, b:e]) <= 1e-4
        assert rel_l2(gM.cpu().numpy(), rM[:, :, b:e]) <= 1e-4


def test_strided_views_are_accepted_by_the_sharded_ops(cuda):
    # a caller that slices the arrays itself (views, not copies) gets the same result
    shape = (1, 64, 64)
    ph = [t.cuda() for t in S.uniform_cluster_photons(5000, 64, 64, seed=32)]
    views = (ph[0][100:4000], ph[1][:, 100:4000], ph[2][:, :, 100:4000], ph[3][:, 100:4000],
             ph[4][100:4000])
    assert not views[1].is_contiguous()
    a = SH.sharded_forward(*views, list(shape), 20)[0]
    b = SH.sharded_forward(*(t.contiguous() for t in views), list(shape), 20)[0]
    torch.cuda.synchronize()
    assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) <= 1e-6
