"""The splat plan's binning, bit for bit against a CPU restatement (``oracle/plan_keys.py``).

Through ``pds_plan_export`` every photon's bucket key and slot are read back after
``pds_plan_f32`` / ``pds_batch_plan_f32``, and checked:

  - the keys equal the CPU restatement's exactly (simulation, channel, screen tile of the
    clamped centre pixel, row class; wide and untouched photons classified identically) with
    the row walk's 6 class bits; with the library default (band walk, 5 class bits, whose
    area classes come from approximate intrinsics) every field above the class;
  - the sorted positions of the tile-path photons are a permutation of [0, n_tile) grouped by
    ascending key: the photons of key k occupy exactly positions [s_k, s_k + count_k) with
    s_k the number of tile-path photons of smaller keys (a counting sort of the CPU keys;
    the order inside one key is not fixed);
  - the wide photons' slots are a permutation of [0, n_wide); untouched photons have none.
"""
import ctypes

import numpy as np
import pytest
import torch

from oracle import plan_keys as PK
from shapefromcaustics_b200 import _lib
from shapefromcaustics_b200 import synthetic as S

pytestmark = pytest.mark.gpu

NONE = 0xFFFFFFFF


def export(ws, n, n_tiles, mpr, cfg):
    bucket = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    slot = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    lib = _lib.lib()
    _lib.check(lib.pds_plan_export(ctypes.c_void_p(ws.data_ptr()), ws.numel(), n, n_tiles, mpr,
                                   ctypes.byref(cfg), ctypes.c_void_p(bucket.data_ptr()),
                                   ctypes.c_void_p(slot.data_ptr()),
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    return (bucket.cpu().numpy().view(np.uint32)[:n].astype(np.int64),
            slot.cpu().numpy().view(np.uint32)[:n].astype(np.int64))


def check_binning(keys_gpu, slots, keys_cpu, n_tiles, class_bits=6):
    """class_bits 6: keys equal exactly; other class bits: equal above the class field, and
    the device's classes in range (the band classes come from approximate intrinsics)."""
    if class_bits == 6:
        assert np.array_equal(keys_gpu, keys_cpu)
    else:
        assert np.array_equal(keys_gpu >> class_bits, keys_cpu >> class_bits)
        sentinel = (keys_gpu >> class_bits) >= n_tiles
        assert np.all(keys_gpu[sentinel] & ((1 << class_bits) - 1) == 0)
    key_big = n_tiles << class_bits
    key_invalid = (n_tiles + 1) << class_bits
    tile = keys_gpu < key_big
    wide = keys_gpu == key_big
    none = keys_gpu == key_invalid
    assert np.all(tile | wide | none)
    n_tile = int(tile.sum())
    # tile path: positions grouped by ascending key
    k = keys_gpu[tile]
    pos = slots[tile]
    assert np.array_equal(np.sort(pos), np.arange(n_tile))
    order = np.argsort(k, kind="stable")
    ks, ps = k[order], pos[order]
    starts = np.searchsorted(ks, ks, side="left")
    ends = np.searchsorted(ks, ks, side="right")
    assert np.all((ps >= starts) & (ps < ends))
    # wide list and untouched photons
    assert np.array_equal(np.sort(slots[wide]), np.arange(int(wide.sum())))
    assert np.all(slots[none] == NONE)
    return n_tile, int(wide.sum()), int(none.sum())


# the library default (band walk, 5 class bits) and the row walk's classes (6 bits)
CONFIGS = [dict(), dict(walk=4, class_bits=6)]


def class_bits_of(kw):
    return kw.get("class_bits", 5)


@pytest.mark.parametrize("kw", CONFIGS)
def test_single_simulation_binning_is_exact(cuda, kw):
    from shapefromcaustics_b200.splatting import SplatPlan
    n, H, W, C = 2 ** 18, 300, 520, 3
    E, X, M, _, R = S.uniform_cluster_photons(n, H, W, seed=40, s_range=(0.3, 9.0))
    g = torch.Generator().manual_seed(41)
    cp = torch.randint(-1, C + 1, (1, n), generator=g)  # some channels out of range
    # some photons off the image entirely
    X[:, :500] = X[:, :500] * 1.5
    ph = (E, X, M, cp, R)
    mpr = 20
    cb = class_bits_of(kw)
    cfg = _lib.config(apron_max=6, **kw)  # footprints wider than 6 px take the wide list
    plan = SplatPlan(*(t.cuda() for t in ph), (C, H, W), mpr, config=cfg)
    n_tiles = C * ((H + 63) // 64) * ((W + 63) // 64)
    kg, sl = export(plan.ws, n, n_tiles, mpr, cfg)
    kc, nt = PK.plan_keys([t.numpy() for t in ph], [(n, (C, H, W))], mpr, apron_max=6,
                          class_bits=cb)
    assert nt == n_tiles
    n_tile, n_wide, n_none = check_binning(kg, sl, kc, n_tiles, cb)
    assert n_tile > 0 and n_wide > 0 and n_none > 0


@pytest.mark.parametrize("kw", CONFIGS)
@pytest.mark.parametrize("mpr", [20, 3])
def test_batch_binning_is_exact(cuda, mpr, kw):
    from shapefromcaustics_b200.splatting import BatchedSplat
    specs = [(40000, (1, 256, 256)), (0, (1, 64, 64)), (120000, (2, 512, 384)),
             (7000, (1, 96, 130)), (300000, (1, 1024, 1024))]
    parts = []
    for s, (n, (C, H, W)) in enumerate(specs):
        ph = S.uniform_cluster_photons(max(n, 1), H, W, seed=50 + s, s_range=(0.4, 6.0))
        ph = tuple(t[..., :n] for t in ph)
        if C > 1:
            ph = (ph[0], ph[1], ph[2],
                  torch.randint(0, C, (1, n), generator=torch.Generator().manual_seed(s)), ph[4])
        parts.append(ph)
    cat = [torch.cat([p[k] for p in parts], dim=-1).contiguous() for k in range(5)]
    cb = class_bits_of(kw)
    b = BatchedSplat(specs, mpr, "cuda:0", config=_lib.config(**kw))
    b.plan(*(t.cuda() for t in cat))
    n = sum(n for n, _ in specs)
    kg, sl = export(b.ws, n, b.n_tiles, mpr, b.cfg)
    kc, nt = PK.plan_keys([t.numpy() for t in cat], specs, mpr, class_bits=cb)
    assert nt == b.n_tiles
    check_binning(kg, sl, kc, b.n_tiles, cb)


def test_binning_past_the_shared_window_on_2048(cuda):
    # 2048^2 at 6 class bits: 65536 buckets, more than the plan's shared histogram window
    # holds (32768), so part of the photons are counted and placed with global atomics
    from shapefromcaustics_b200.splatting import SplatPlan
    n, H, W = 2 ** 19, 2048, 2048
    ph = S.caustic_curve_photons(n, H, W, seed=42)
    cfg = _lib.config(walk=4, class_bits=6)
    plan = SplatPlan(*(t.cuda() for t in ph), (1, H, W), 20, config=cfg)
    n_tiles = (H // 64) * (W // 64)
    kg, sl = export(plan.ws, n, n_tiles, 20, plan.cfg)
    kc, _ = PK.plan_keys([t.numpy() for t in ph], [(n, (1, H, W))], 20)
    check_binning(kg, sl, kc, n_tiles)
