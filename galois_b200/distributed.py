"""Multi-GPU betweenness centrality: the sources are sharded over the ranks
and one all-reduce sums the partial centralities.

Brandes BC over a set of sources is a sum of per-source dependency vectors
(LevelStructs.h:147-183 accumulates them into one bc array), so ranks that
each own a disjoint subset of the sources need no communication until the
end: a single SUM all-reduce of the n-vector.  Every other kernel of this
package runs one replica per GPU (no exchange step exists on its path).

One process per GPU; the process group is the caller's (NCCL on GPUs, gloo
for host tests).
"""
from __future__ import annotations

import numpy as np


def shard_sources(sources, rank: int, world: int) -> np.ndarray:
    """The sources owned by `rank`: every world-th source starting at rank
    (strided, so each rank gets a similar mix of early and late sources)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    return np.ascontiguousarray(np.asarray(sources, dtype=np.uint32)[rank::world])


def bc_sharded(graph, sources, out, batch: int = 64, group=None):
    """Brandes BC of `graph` over `sources` summed across the ranks of `group`.

    `graph` is a DeviceGraph (or anything with its bc(sources, batch, out)
    method); `out` is this rank's float32 tensor of n entries (on the rank's
    GPU for NCCL).  Every rank must call with the same `sources`; on return
    every rank holds the full result in `out`."""
    import torch.distributed as dist

    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    mine = shard_sources(sources, rank, world)
    if mine.size:
        graph.bc(mine, batch=batch, out=out)
    else:
        out.zero_()
    dist.all_reduce(out, op=dist.ReduceOp.SUM, group=group)
    return out
