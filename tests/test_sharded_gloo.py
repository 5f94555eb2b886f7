"""The sharded path's exchange on the CPU (world_size 3, gloo): shard ranges
cover every row group once in rank order, and rank 0 receives every rank's
partial bytes in rank order whatever order the ranks finish in. The GPU merge
itself is tested in tests/test_gpu_sharded.py."""
from __future__ import annotations

import json
import os
import socket
import time

import pytest
import torch.multiprocessing as mp

from vexq_b200.sharded import shard_range


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("n_rg,world", [(0, 1), (1, 3), (7, 3), (49, 8), (1000, 7)])
def test_shard_ranges_partition_the_row_groups(n_rg, world):
    seen = []
    prev_end = 0
    for r in range(world):
        s, e = shard_range(n_rg, r, world)
        assert s == prev_end and e >= s and e - s in (n_rg // world, n_rg // world + 1)
        seen += list(range(s, e))
        prev_end = e
    assert seen == list(range(n_rg))
    with pytest.raises(ValueError):
        shard_range(n_rg, world, world)


def _worker(rank: int, world: int, port: int, out_dir: str):
    import datetime

    import torch.distributed as dist

    from vexq_b200.sharded import gather_partials
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        time.sleep(0.05 * (world - rank))  # the last rank finishes first
        part = bytes([rank]) * (100 + rank) + b"end"
        got = gather_partials(part, rank, world)
        with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
            json.dump(None if got is None else [g.hex() for g in got], f)
    finally:
        dist.destroy_process_group()


def test_gather_in_rank_order(tmp_path):
    world = 3
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    r0 = json.load(open(tmp_path / "r0.json"))
    assert [bytes.fromhex(h) for h in r0] == [bytes([r]) * (100 + r) + b"end" for r in range(world)]
    for r in range(1, world):
        assert json.load(open(tmp_path / f"r{r}.json")) is None
