"""Host logic of the multi-GPU benchmark path, run as two gloo ranks on the CPU.

On N GPUs every rank splats its own independently seeded batch of simulations (the
simulations shard with no data-path exchange); the only cross-rank steps are the barrier
around the timed region and the max / sum reductions of the step time and photon count.
"""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import datetime
    import bench
    from shapefromcaustics_b200 import synthetic as S
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        r, w, l = bench.dist_env()
        bench.barrier(w)
        mx = bench.max_over_ranks(float(rank + 1), w, "cpu")
        sm = bench.sum_over_ranks(float(10 * (rank + 1)), w, "cpu")
        specs = S.batch_specs(64, seed=1000 + rank)
        ref = bench.run_reference_cpu(type("A", (), {"workload": "uniform1m", "steps": 1,
                                                     "warmup": 0, "ref_sample": 2 ** 12})(),
                                      r, w) if rank == 1 else "skipped"
        q.put((rank, r, w, mx, sm, sum(n for n, _ in specs), ref))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_and_shard():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    for rank, r, w, mx, sm, n, ref in out:
        assert r == rank and w == 2
        assert mx == 2.0 and sm == 30.0
    # ranks draw different batches (independent seeds)
    assert out[0][5] != out[1][5]
    # the reference arm runs on rank 0 only; other ranks return nothing
    assert out[1][6] is None


def _sharded_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import numpy as np
    from oracle import oracle as O
    from shapefromcaustics_b200 import sharded as SH
    from shapefromcaustics_b200 import synthetic as S
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        shape = (1, 96, 80)
        ph = S.uniform_cluster_photons(3001, 96, 80, seed=21, sigma=6.0)
        local = SH.shard_photons(*ph, rank, world)
        # the CUDA ops take contiguous arrays only
        assert all(t.is_contiguous() for t in local)

        def oracle_fwd(E, X, M, C, R, size, mpr):
            img = O.forward(*[t.numpy() for t in (E, X, M, C, R)], tuple(size), mpr)
            return [torch.from_numpy(np.ascontiguousarray(img))]

        def oracle_bwd(G, E, X, M, C, R, mpr):
            return [torch.from_numpy(np.ascontiguousarray(a)) for a in
                    O.backward(G.numpy(), *[t.numpy() for t in (E, X, M, C, R)], mpr)]

        img = SH.sharded_forward(*local, list(shape), 20, splat=oracle_fwd)[0]
        G = S.upstream_grad(shape, seed=5).double()
        grads = SH.sharded_backward(G, *local, 20, splat_backward=oracle_bwd)
        q.put((rank, img.numpy(), [g.numpy() for g in grads], SH.shard_range(3001, rank, world)))
    finally:
        dist.destroy_process_group()


def test_photon_sharded_simulation_sums_partial_images():
    """One simulation split by photons over two gloo ranks: the all-reduced partial images
    equal the whole simulation's image, and each rank's gradients equal its slice of the whole
    simulation's gradients (the oracle stands in for the GPU splat on the CPU)."""
    import numpy as np
    from oracle import oracle as O
    from shapefromcaustics_b200 import synthetic as S
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=180) for _ in procs], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shape = (1, 96, 80)
    ph = [t.numpy() for t in S.uniform_cluster_photons(3001, 96, 80, seed=21, sigma=6.0)]
    full = O.forward(*ph, shape, 20)
    G = S.upstream_grad(shape, seed=5).double().numpy()
    gE, gX, gM = O.backward(G, *ph, 20)
    assert [r[3] for r in out] == [(0, 1501), (1501, 3001)]
    for rank, img, (lE, lX, lM), (b, e) in out:
        assert np.linalg.norm(img - full) <= 1e-12 * np.linalg.norm(full)
        assert np.array_equal(lE, gE[b:e])
        assert np.array_equal(lX, gX[:, b:e])
        assert np.array_equal(lM, gM[:, :, b:e])
