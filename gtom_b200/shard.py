"""Data-parallel insertion across ranks (one process per GPU).

Slices are independent until they meet in the Fourier accumulators, so the
multi-GPU form of d_rlnBackproject shards the slice batch across ranks, lets
every rank insert its share into a private pair of accumulators, and sums
the partial accumulators with ONE all-reduce.  To make that a single
collective the complex data accumulator and the real weight accumulator are
views into one contiguous float buffer: [re, im] * nvox followed by nvox
weights.  The projector needs no exchange at all (every rank holds the
reference volume and projects its own slices).

Around them: the reference volume the projector reads is replicated with one
broadcast per reference update (broadcast_reference), and independent
reconstructions (half-maps, classes, sub-tomograms) are spread over ranks
whole (volumes_for_rank): one volume's gridding is not split across GPUs,
it runs as a replica on its rank.

The reference has no multi-GPU path for these functions; callers of
gtom's d_rlnBackproject (src/Relion/Backproject.cu:22-76) that split their
particle stacks across devices sum the volumes on the host.
"""
from __future__ import annotations

import torch


def slice_range(total: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous share of `total` slices for `rank`: (first, count).
    Shares differ by at most one slice; the first total % world ranks take
    the extra ones."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    if total < 0:
        raise ValueError("negative slice count")
    base, extra = divmod(total, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def volumes_for_rank(nvolumes: int, rank: int, world: int) -> list[int]:
    """The independent volumes (half-maps, classes, sub-tomograms) that
    `rank` reconstructs: volume i belongs to rank i % world, so every volume
    has exactly one owner and the ranks' counts differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    if nvolumes < 0:
        raise ValueError("negative volume count")
    return list(range(rank, nvolumes, world))


def broadcast_reference(volft: torch.Tensor, src: int = 0, group=None) -> None:
    """Replicates the reference volume the projector reads (the decentred
    half-complex array) from rank `src` to every rank, in place: the one
    exchange the projector needs, once per reference update.  A no-op
    without an initialised process group or with one rank."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return
    if dist.get_world_size(group) == 1:
        return
    buf = torch.view_as_real(volft) if volft.is_complex() else volft
    dist.broadcast(buf, src=src, group=group)


class Accumulators:
    """A complex64 data accumulator and a float32 weight accumulator of
    `nvox` voxels each, laid out back to back in one float32 buffer so that
    their cross-rank sum is one collective."""

    def __init__(self, nvox: int, device):
        self.nvox = int(nvox)
        self.buffer = torch.zeros(3 * self.nvox, dtype=torch.float32, device=device)
        self.data = torch.view_as_complex(self.buffer[:2 * self.nvox].view(self.nvox, 2))
        self.weights = self.buffer[2 * self.nvox:]

    def zero_(self) -> "Accumulators":
        self.buffer.zero_()
        return self

    def all_reduce(self, group=None) -> None:
        """Sums the accumulators of all ranks in place (every rank ends with
        the full sums).  A no-op without an initialised process group or
        with one rank."""
        import torch.distributed as dist
        if not dist.is_available() or not dist.is_initialized():
            return
        if dist.get_world_size(group) == 1:
            return
        dist.all_reduce(self.buffer, op=dist.ReduceOp.SUM, group=group)
