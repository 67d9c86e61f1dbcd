"""Multi-GPU split of the assembly: one process per GPU, stencils sharded by
contiguous node ranges, no collective on the data path.

Every stencil is independent, so rank r assembles the stencils of its node
range [first, first + count) against the whole node set. The one exchange
is the node coordinates (16 bytes per node), replicated from rank 0 by a
broadcast (NCCL over NVLink / NVSwitch on GPUs, gloo on CPU); every rank then
runs the k-NN search and the assembly on its own HBM. The CSR rows stay
sharded; ``gather_rows`` assembles them on every rank when a caller wants the
whole operator.

The reference has no multi-process code; this follows the split it would
take (contiguous ranges, ideally after a Morton renumbering so that the
neighbour gathers stay local).
"""
from __future__ import annotations

import torch


def node_range(n: int, world: int, rank: int):
    """Contiguous, balanced range of rank `rank`: (first, count)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def replicate_nodes(x: torch.Tensor, y: torch.Tensor, src: int = 0, group=None):
    """Broadcast the node coordinates from rank `src` to every rank (in place)."""
    import torch.distributed as dist
    dist.broadcast(x, src=src, group=group)
    dist.broadcast(y, src=src, group=group)
    return x, y


def gather_rows(rows: torch.Tensor, n: int, k: int, world: int, group=None) -> torch.Tensor:
    """All-gather fixed-width row blocks (rank r holds node_range(n, world,
    r) rows of k values) into the full n*k array on every rank."""
    import torch.distributed as dist
    counts = [node_range(n, world, r)[1] for r in range(world)]
    cmax = max(counts)
    pad = torch.zeros(cmax * k, dtype=rows.dtype, device=rows.device)
    pad[: rows.numel()] = rows
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad, group=group)
    return torch.cat([b[: c * k] for b, c in zip(bufs, counts)])


def assemble_shard(ctx, desc, x: torch.Tensor, y: torch.Tensor, k: int, rank: int, world: int,
                   period=None):
    """k-NN stencils and weights of this rank's node range, on this rank's
    GPU. Returns (first, count, ja_rows, [values_rows...])."""
    import rbf_b200 as R
    n = x.numel()
    first, count = node_range(n, world, rank)
    nrhs = R.num_rhs(desc.ops, desc.nc)
    ja = torch.empty(max(count, 1) * k, dtype=torch.int32, device=x.device)
    vals = [torch.empty(max(count, 1) * k, dtype=torch.float64, device=x.device)
            for _ in range(nrhs)]
    info = torch.empty(max(count, 1), dtype=torch.int32, device=x.device)
    if count:
        xq, yq = x[first:first + count].contiguous(), y[first:first + count].contiguous()
        ctx.knn_query(x, y, xq, yq, k, ja, period=period)
        ctx.assemble_range(desc, first, count, x, y, k, ja, vals, info)
    return first, count, ja[: count * k], [v[: count * k] for v in vals]
