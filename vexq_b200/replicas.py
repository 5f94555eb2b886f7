"""Replica execution across ranks: one process per GPU, no data-path collective.

The hot path shards by row group with no exchange (exec/parallel.go:18-36
hands independent morsels to workers), so every rank owns its own tables and
runs the same step. The timed region is bracketed by barriers on both sides
and the job's time is the maximum over ranks; the whole-job rate is the sum
of all ranks' bytes over that time (weak scaling). The helpers take their
timers and process group as arguments so the same code runs under NCCL on
GPUs and under gloo on the CPU.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Tuple


def run_timed(step: Callable[[], object], steps: int, warmup: int, start: Callable[[], None],
              stop: Callable[[], float], barrier: Optional[Callable[[], None]] = None) -> Tuple[float, List[object]]:
    """max(warmup, 3) untimed steps, barrier, start timer, exactly `steps`
    steps, stop timer (milliseconds), barrier. Returns (ms, per-step results)."""
    for _ in range(max(warmup, 3)):
        step()
    if barrier:
        barrier()
    start()
    out = [step() for _ in range(steps)]
    ms = stop()
    if barrier:
        barrier()
    return ms, out


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Maximum of a per-rank float over the process group (the value itself
    when there is no group or one rank)."""
    if dist is None or not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate_gbs(bytes_per_rank_step: int, world: int, max_ms_per_step: float) -> float:
    """Whole-job GB/s: every rank's bytes of one step over the slowest rank's step time."""
    return bytes_per_rank_step * world / (max_ms_per_step / 1e3) / 1e9
