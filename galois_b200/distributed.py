"""Multi-GPU sharding of the two batched kernels over independent units.

* Brandes BC: the sources are sharded over the ranks and one all-reduce sums
  the partial centralities.  BC over a set of sources is a sum of per-source
  dependency vectors (LevelStructs.h:147-183 accumulates them into one bc
  array), so ranks that each own a disjoint subset of the sources need no
  communication until the end: a single SUM all-reduce of the n-vector.
* Personalised PageRank with its adjoint: the teleport columns are sharded
  (blocks of whole multiples of 4, the batched kernels' unit).  Columns are
  independent in the forward and the adjoint solve; the gradient with
  respect to the shared arc weights is a sum over columns, so one SUM
  all-reduce of the m-vector is the only exchange.
Every other kernel of this package runs one replica per GPU (no exchange
step exists on its path).

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


def shard_columns(B: int, rank: int, world: int) -> tuple[int, int]:
    """[begin, end) of the teleport columns owned by `rank`: contiguous
    blocks whose sizes are multiples of 4 (the batched PPR kernels take 1 or
    a multiple of 4 columns), as even as that allows; a lone column (B = 1)
    goes to rank 0.  A rank may own none."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    if B <= 0:
        return 0, 0
    if B % 4:
        if B != 1:
            raise ValueError("B must be 1 or a multiple of 4")
        return (0, 1) if rank == 0 else (0, 0)
    groups = B // 4
    per, extra = divmod(groups, world)
    g0 = rank * per + min(rank, extra)
    g1 = g0 + per + (1 if rank < extra else 0)
    return 4 * g0, 4 * g1


def ppr_sharded(graph, teleport, w, c, alpha: float = 0.85, tol: float = 1e-7, max_iter: int = 1000, group=None,
                solve=None):
    """Forward and adjoint of the batched personalised PageRank with
    loss = sum(c * x), the columns of `teleport` ([n, B]) sharded over the
    ranks of `group`.

    Every rank passes the same full `teleport`, `c` ([n, B]) and `w` (arc
    weights, [m]); it solves only its own columns and returns
    (x_local, (begin, end), grad_teleport_local, grad_w, loss), where
    grad_w is the full gradient of the whole loss with respect to w (summed
    over every rank's columns by one all-reduce) and loss the whole loss.
    `solve(graph, T, w, alpha, tol, max_iter)` defaults to
    galois_b200.ppr.ppr (the differentiable GPU solve)."""
    import torch
    import torch.distributed as dist

    if solve is None:
        from .ppr import ppr as solve
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    b0, b1 = shard_columns(teleport.shape[1], rank, world)
    wl = w.detach().clone().requires_grad_(True)
    if b1 > b0:
        tl = teleport[:, b0:b1].detach().contiguous().requires_grad_(True)
        x = solve(graph, tl, wl, alpha, tol, max_iter)
        loss = (c[:, b0:b1] * x).sum()
        loss.backward()
        gw = wl.grad
        gt = tl.grad
        x = x.detach()
    else:
        x = teleport[:, 0:0]
        gt = teleport[:, 0:0]
        loss = torch.zeros((), dtype=w.dtype, device=w.device)
        gw = torch.zeros_like(w)
    gw = gw.contiguous()
    dist.all_reduce(gw, op=dist.ReduceOp.SUM, group=group)
    total = loss.detach().reshape(1).clone()
    dist.all_reduce(total, op=dist.ReduceOp.SUM, group=group)
    return x, (b0, b1), gt, gw, total[0]
