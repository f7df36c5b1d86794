"""Autotuner for the splat kernels' launch configuration.

Times candidate ``pds_config`` values (screen-tile edge, sorted photons per work chunk,
footprint-class sort bits, pixel walk, resident CTAs per SM, warp-cooperative splat of large
footprints) on the caller's actual workload with CUDA events, and keeps the fastest per workload signature (photon count
and image sizes, bucketed); the first candidate is the library default, which wins ties. The
reference has a single fixed launch shape (512 threads per photon block,
``photon_differentials.cu:120``); here the best tile and chunk depend on footprint sizes and
photon density, so they are measured rather than fixed.
"""
import itertools
import math

import torch

from . import _lib

__all__ = ["DEFAULT", "CANDIDATES", "signature", "pick", "tune_batch", "cached"]

# the library default first; then tile, class bits, walk, CTAs per SM and the cooperative
# splat in all combinations, and the default with smaller and larger work chunks (sorted
# photons a CTA takes at a time). min_blocks 0 is the library's choice per direction (3 CTAs
# an SM for the forward, 4 for the backward); 4 sets both.
DEFAULT = dict(tile=64, chunk=2048, class_bits=5, walk=3, min_blocks=0, coop_radius=-1)
CANDIDATES = [dict(tile=t, chunk=2048, class_bits=b, walk=w, min_blocks=m, coop_radius=k)
              for t, b, w, m, k in itertools.product((64, 32), (5, 3), (3, 1), (0, 4), (-1, 8))]
CANDIDATES += [dict(DEFAULT, chunk=c) for c in (1024, 4096)]
# the padded-row walk with its row classes, at both tile sizes and CTA counts
CANDIDATES += [dict(tile=t, chunk=2048, class_bits=6, walk=4, min_blocks=m, coop_radius=-1)
               for t, m in itertools.product((64, 32), (0, 4))]

_cache = {}


def signature(specs, max_pixel_radius):
    """Bucketed description of a workload: log2 of the photon count, the image sizes."""
    n = sum(n for n, _ in specs)
    sizes = tuple(sorted({tuple(int(v) for v in shape) for _, shape in specs}))
    return (int(math.log2(max(n, 1))), sizes, int(max_pixel_radius), len(specs) > 1)


def cached(specs, max_pixel_radius):
    return _cache.get(signature(specs, max_pixel_radius))


def _time_step(batch, photons, out, gflat, grads, reps, stream):
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        ev0.record(stream)
        for _ in range(reps):
            batch.plan(*photons)
            batch.forward(out)
            batch.backward(gflat, grads)
        ev1.record(stream)
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1) / reps


def _measure(batch, photons, out, gflat, grads, reps, stream, min_ms=20.0, rounds=3):
    """ms per step: a warm-up step, then `rounds` timings of at least `reps` steps and about
    `min_ms` of work each; the fastest round (the least disturbed) counts."""
    t = _time_step(batch, photons, out, gflat, grads, 1, stream)
    reps = max(reps, min(200, int(math.ceil(min_ms / max(t, 1e-3)))))
    return min(_time_step(batch, photons, out, gflat, grads, reps, stream)
               for _ in range(rounds))


def pick(timed, margin=0.02):
    """The winner of ``timed``, a list of ``(config, ms)`` in candidate order: the first entry
    (the library default) unless another is faster than it by more than ``margin`` (a
    fraction), in which case the fastest of those. ``None`` for an empty list."""
    if not timed:
        return None
    first_cfg, first_ms = timed[0]
    best, best_ms = first_cfg, first_ms
    for c, ms in timed[1:]:
        if ms < best_ms and ms < first_ms * (1.0 - margin):
            best, best_ms = c, ms
    return best


def tune_batch(specs, photons, gflat, max_pixel_radius, device, candidates=None, reps=3,
               verbose=False, margin=0.02):
    """Times every candidate on ``BatchedSplat(specs)`` with the given photons and upstream
    gradient; returns ``(best_config_dict, {config_key: ms})`` and caches the winner. The first
    candidate (the library default) is kept unless another is faster by more than
    ``margin``."""
    from .splatting import BatchedSplat
    candidates = candidates or CANDIDATES
    stream = torch.cuda.Stream(device)
    results = {}
    timed = []
    grads = tuple(torch.empty_like(t) for t in photons[:3])
    out = None
    for c in candidates:
        cfg = _lib.config(**c)
        try:
            batch = BatchedSplat(specs, max_pixel_radius, device, config=cfg)
        except _lib.PdsError:
            continue
        if out is None:
            out = torch.empty(batch.image_elems, device=device)
        ms = _measure(batch, photons, out, gflat, grads, reps, stream)
        key = tuple(sorted(c.items()))
        results[key] = ms
        timed.append((c, ms))
        if verbose:
            print(f"autotune {c}: {ms:.3f} ms")
        del batch
    best = pick(timed, margin)
    _cache[signature(specs, max_pixel_radius)] = best
    return best, results
