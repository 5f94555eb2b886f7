"""One query split across GPUs by row group: one process per GPU, each
holding the whole table (the same dictionaries, so group keys agree), rank r
scanning row groups [r·n/N, (r+1)·n/N). Each rank's run yields a partial —
its groups unfinished (vexq_plan_run_partial); the partials are gathered to
rank 0 in rank order, the one exchange the path has, and merged there
(vexq_partial_merge): ParallelHashAggregate's partial aggregates and
mergePartialAgg (exec/parallel.go:124-210, 237-314) with ranks in place of
workers. A join shards its probe side; every rank builds the whole build
side. The gather goes through torch.distributed, so the same code runs under
NCCL on GPUs and under gloo on the CPU."""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple


def shard_range(n_rg: int, rank: int, world: int) -> Tuple[int, int]:
    """Row groups [start, end) of `rank`'s shard: contiguous, in rank order,
    sizes differing by at most one, together every row group once."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank outside the world")
    return (n_rg * rank) // world, (n_rg * (rank + 1)) // world


def gather_partials(part: bytes, rank: int, world: int, group=None) -> Optional[List[bytes]]:
    """Every rank's partial on rank 0, in rank order (None elsewhere)."""
    import torch.distributed as dist
    if world == 1:
        return [part]
    out: Optional[List[object]] = [None] * world if rank == 0 else None
    dist.gather_object(part, out, dst=0, group=group)
    return out  # type: ignore[return-value]


def run_sharded(op, n_rg: int, rank: int, world: int, group=None):
    """The finished result on rank 0 (None on the other ranks)."""
    rs, re = shard_range(n_rg, rank, world)
    parts = gather_partials(op.run_partial(rs, re), rank, world, group)
    return op.merge_partials(parts) if rank == 0 else None


def merge_in_rank_order(op, parts: Sequence[bytes]):
    """The merge rank 0 runs, for callers that gathered the bytes themselves."""
    return op.merge_partials(list(parts))
