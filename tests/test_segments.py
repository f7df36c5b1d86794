"""The tile kernels' walk over the plan's sorted photons, emulated on the CPU.

fwd_tiles_kernel and bwd_tiles_kernel (csrc/pds_splat.cu) take chunks of sorted positions and
split each batch of NT positions into runs of one screen tile ("segments"), found from the
plan's bucket starts: the chunk's first tile comes from chunk_tile_kernel (csrc/pds_plan.cu),
the next non-empty tile from a doubling search then a bisection. This restates that control
flow line for line and checks, over random bucket tables with empty tiles and chunk
boundaries inside tiles, that every position is handled exactly once, by the tile whose range
holds it, within the kernels' cap of NT + 1 passes per batch.
"""
import numpy as np
import pytest


def chunk_tile(start, cb, n_tiles, p):
    lo, hi = 0, n_tiles - 1
    while lo < hi:
        mid = (lo + hi + 1) >> 1
        if start[mid << cb] <= p:
            lo = mid
        else:
            hi = mid - 1
    return lo


def tile_end(start, cb, t):
    return int(start[(t + 1) << cb])


def next_segment(start, cb, n_tiles, tile, end):
    p, t, last = end, tile, n_tiles - 1
    k, steps = 1, 0
    while t + k < last and tile_end(start, cb, t + k) <= p:
        k <<= 1
        steps += 1
        assert steps < 64
    lo, hi = t + (k >> 1) + 1, min(t + k, last)
    while lo < hi:
        mid = (lo + hi) >> 1
        if tile_end(start, cb, mid) > p:
            hi = mid
        else:
            lo = mid + 1
    return lo, p, tile_end(start, cb, lo)


def walk(counts, cb, n_tiles, chunk, nt):
    start = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    n_tile = int(start[-1])
    owner = np.full(n_tile, -1)
    nchunks = (n_tile + chunk - 1) // chunk
    for c in range(nchunks):
        p0, p1 = c * chunk, min(c * chunk + chunk, n_tile)
        tile = chunk_tile(start, cb, n_tiles, p0)
        begin, end = p0, tile_end(start, cb, tile)
        for base in range(p0, p1, nt):
            bend = min(base + nt, p1)
            for _ in range(nt + 1):
                for i in range(max(base, begin), min(bend, end)):
                    assert owner[i] == -1
                    owner[i] = tile
                if end >= bend:
                    break
                tile, begin, end = next_segment(start, cb, n_tiles, tile, end)
            else:
                raise AssertionError("segment loop reached its pass cap")
    return start, owner


@pytest.mark.parametrize("seed", range(12))
def test_every_sorted_photon_is_walked_once_by_its_tile(seed):
    rng = np.random.default_rng(seed)
    cb = int(rng.integers(0, 4))
    n_tiles = int(rng.integers(1, 60))
    nb = n_tiles << cb
    # sparse tables: many empty buckets and tiles, some heavy ones
    counts = rng.integers(0, 3, nb) * (rng.random(nb) < 0.3)
    heavy = rng.integers(0, nb, 3)
    counts[heavy] += rng.integers(0, 900, 3)
    if seed % 3 == 0:
        counts[: nb // 2] = 0  # leading empty tiles
    if counts.sum() == 0:
        counts[-1] = 5
    chunk = int(rng.choice([256, 512]))
    nt = int(rng.choice([32, 64, 256]))
    start, owner = walk(counts, cb, n_tiles, chunk, nt)
    assert np.all(owner >= 0)
    tiles_of = np.searchsorted(start[:: 1 << cb][1:], np.arange(len(owner)), side="right")
    assert np.array_equal(owner, tiles_of)
