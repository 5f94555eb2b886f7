"""Multi-rank replica logic on the CPU (world_size 2, gloo): barriers around
the timed region, the maximum over ranks, the whole-job rate, and that every
rank's result is the one its own shard gives in a single process. The step
is the oracle's aggregate over a rank-seeded shard, the CPU stand-in for a
rank's GPU step."""
from __future__ import annotations

import json
import os
import socket
import time

import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _shard_rows(rank: int):
    from oracle import refcpu as R
    from vexq_b200 import datagen as D, workloads as W
    t = D.lineitem(20_000, seed=100 + rank, rg_rows=4096)
    return R.agg(R.RefTable(t), W.q1_plan(), workers=0).rows()


def _worker(rank: int, world: int, port: int, out_dir: str):
    import datetime

    import torch.distributed as dist

    from vexq_b200.replicas import job_rate_gbs, max_over_ranks, run_timed
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rows = []
        t0 = [0.0]

        def step():
            time.sleep(0.02 * (rank + 1))  # rank 1 is the slow one
            rows.append(_shard_rows(rank))
            return len(rows[-1])

        def start():
            t0[0] = time.perf_counter()

        def stop():
            return (time.perf_counter() - t0[0]) * 1e3

        ms, out = run_timed(step, 2, 3, start, stop, dist.barrier)
        mx = max_over_ranks(ms, dist)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"ms": ms, "max": mx, "steps": len(out), "calls": len(rows),
                       "rows": [list(map(repr, r)) for r in rows[-1]],
                       "rate": job_rate_gbs(1_000_000, world, mx / 2)}, f)
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas(tmp_path):
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    r = [json.load(open(tmp_path / f"rank{k}.json")) for k in range(2)]
    assert all(x["steps"] == 2 and x["calls"] == 5 for x in r)  # 3 warm-up + 2 timed
    assert r[0]["max"] == r[1]["max"] == max(r[0]["ms"], r[1]["ms"])
    assert r[1]["ms"] > r[0]["ms"]  # the slow rank sets the job time
    assert abs(r[0]["rate"] - 1_000_000 * 2 / (r[0]["max"] / 2 / 1e3) / 1e9) < 1e-9
    for k in range(2):  # replicas are independent: each equals its shard alone
        assert r[k]["rows"] == [list(map(repr, row)) for row in _shard_rows(k)]
    assert r[0]["rows"] != r[1]["rows"]
