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
