"""One simulation sharded by photons over the ranks of a process group.

A simulation too large for one GPU (or one whose forward should finish sooner) splits its
photons into contiguous shards, one per rank. Every rank splats its shard into a full-size
partial image and one all-reduce (sum) turns the partial images into the simulation's image on
every rank: the reference's forward is a plain sum over photons
(``photon_differentials.cu:106-110``), so the sum of the shards' images is the image. The
backward needs no exchange: every rank holds the whole upstream gradient and computes the
gradients of its own photons (``photon_differentials.cu:136-221`` reads only the photon and the
gradient image).

Simulations that are already independent (the batched Landweber loop) shard by simulation
with no collective at all; this module is for the single large simulation.
"""
import torch
import torch.distributed as dist

from . import splatting

__all__ = ["shard_range", "shard_photons", "sharded_forward", "sharded_backward"]


def shard_range(n, rank, world):
    """Contiguous photon range [begin, end) of ``rank``: the first ``n % world`` ranks take
    one photon more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a group of {world}")
    base, extra = divmod(int(n), world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def shard_photons(Ep, xp, Mp, cp, radius, rank, world):
    """This rank's slice of the reference's photon arrays, as contiguous tensors.

    The slice of a ``[2, N]`` or ``[2, 3, N]`` array along its photon axis is a strided view;
    the splat ops take contiguous arrays only (``PyOptix/utils.hpp:37-41``), so the rows are
    copied into this rank's own ``[2, n]`` / ``[2, 3, n]`` arrays (``Ep`` and ``radius``
    slices are contiguous already and stay views)."""
    b, e = shard_range(Ep.shape[0], rank, world)
    return (Ep[b:e].contiguous(), xp[:, b:e].contiguous(), Mp[:, :, b:e].contiguous(),
            cp[:, b:e].contiguous(), radius[b:e].contiguous())


def sharded_forward(Ep, xp, Mp, cp, radius, output_size, max_pixel_radius, group=None,
                    splat=None):
    """Forward of this rank's photon shard, summed over the group: every rank returns the
    image of all shards (``[image]``, as ``pds_forward``).

    ``splat`` replaces ``pds_forward`` (same signature); the default is the CUDA op."""
    splat = splat or splatting.pds_forward
    Ep, xp, Mp, cp, radius = (t.contiguous() for t in (Ep, xp, Mp, cp, radius))
    img = splat(Ep, xp, Mp, cp, radius, output_size, max_pixel_radius)[0]
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(img, op=dist.ReduceOp.SUM, group=group)
    return [img]


def sharded_backward(grad_pds, Ep, xp, Mp, cp, radius, max_pixel_radius, splat_backward=None):
    """Gradients of this rank's photon shard from the (replicated) upstream gradient; no
    exchange. ``splat_backward`` replaces ``pds_backward`` (same signature)."""
    fn = splat_backward or splatting.pds_backward
    Ep, xp, Mp, cp, radius = (t.contiguous() for t in (Ep, xp, Mp, cp, radius))
    return fn(grad_pds.contiguous(), Ep, xp, Mp, cp, radius, max_pixel_radius)
