"""Multi-GPU runs: one process per GPU, each transporting a disjoint range of
packet ids, then one sum-reduce of the FP64 tallies.

Packets are independent given the counter RNG keyed (seed, instance, packet id),
so a run over G ranks is the single-GPU run split by packet id: the tallies
agree up to the order of FP64 additions and the event counters exactly.  The
reference's analogue is the `mpi_reduce` of its `finalise`
(src/kernelsMod.f90:578-583).  No collective is needed during transport.
"""
from __future__ import annotations

from typing import Callable


def shard_range(nphotons: int, world: int, rank: int) -> tuple[int, int]:
    """Packet ids [first, first + count) of `rank`: contiguous, sizes differing by at
    most one, covering [0, nphotons) exactly once over all ranks."""
    if world < 1 or not 0 <= rank < world or nphotons < 0:
        raise ValueError("shard_range: need world >= 1, 0 <= rank < world, nphotons >= 0")
    base, extra = divmod(nphotons, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def run_sharded(run_range: Callable[[int, int], dict | None], nphotons: int, tallies: list, *,
                counters=None, group=None, dst: int | None = 0) -> tuple[int, int]:
    """Runs this rank's packet range and sums the tallies over the ranks.

    run_range(first, count) transports packets [first, first + count) and adds
    their tallies into the tensors of `tallies` (e.g. a Transport.run_device
    call into device buffers).  `counters` (an int64 tensor of event counts) is
    summed too.  dst=None all-reduces; otherwise the sums land on rank `dst`.
    Returns this rank's (first, count)."""
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    first, count = shard_range(nphotons, world, rank)
    if count:
        run_range(first, count)
    if world > 1:
        for t in list(tallies) + ([counters] if counters is not None else []):
            if dst is None:
                dist.all_reduce(t, group=group)
            else:
                dist.reduce(t, dst, group=group)
    return first, count
