"""View sharding of one MLEM reconstruction across ranks (one process per GPU).

Every rank owns a contiguous range of views: it forward projects them, forms
their ratios and back projects them into a partial Ht.  The partial images are
summed across ranks in a fixed rank order -- all-to-all of volume slices, an
ordered local sum, all-gather -- so the result is bit-identical on every rank
and from run to run (a library all-reduce may pick its reduction order per
call).  Then every rank applies the same update.  Over NCCL on NVLink this is
4*V bytes out and in per rank per iteration (67 MB for a 256^3 volume).
"""
from __future__ import annotations

from typing import Callable

import torch
import torch.distributed as dist


def view_range(nviews: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous split of nviews over world ranks: (first, count) of `rank`."""
    base, rem = divmod(nviews, world)
    first = rank * base + min(rank, rem)
    return first, base + (1 if rank < rem else 0)


def ordered_sum_(t: torch.Tensor, group=None) -> torch.Tensor:
    """In-place sum of `t` over all ranks, accumulated in rank order 0..N-1."""
    world = dist.get_world_size(group)
    if world == 1:
        return t
    flat = t.reshape(-1)
    n = flat.numel()
    per = (n + world - 1) // world
    padded = torch.zeros(per * world, dtype=t.dtype, device=t.device)
    padded[:n] = flat
    recv = torch.empty_like(padded)
    dist.all_to_all_single(recv, padded, group=group)  # recv[r*per:(r+1)*per] = rank r's copy of my slice
    parts = recv.view(world, per)
    mine = parts[0].clone()
    for r in range(1, world):
        mine += parts[r]
    gathered = torch.empty_like(padded)
    if hasattr(dist, "all_gather_into_tensor") and t.is_cuda:
        dist.all_gather_into_tensor(gathered, mine, group=group)
    else:
        chunks = list(gathered.view(world, per).unbind(0))
        dist.all_gather(chunks, mine, group=group)
        gathered = torch.cat(chunks)
    flat.copy_(gathered[:n])
    return t


def sharded_iteration(nviews: int, forward: Callable[[int, int], None],
                      backward: Callable[[int, int, torch.Tensor], None],
                      update: Callable[[torch.Tensor], None], ht: torch.Tensor, group=None) -> None:
    """One MLEM iteration with views split over the ranks of `group`.

    forward(first, count): ratios of the local views; backward(first, count,
    ht): partial back projection into ht (overwrite); update(ht): the
    multiplicative update with the summed ht."""
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    first, count = view_range(nviews, rank, world)
    forward(first, count)
    backward(first, count, ht)
    if world > 1:
        ordered_sum_(ht, group)
    update(ht)
