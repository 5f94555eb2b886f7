"""CPU test of bench.py's reference arm (`--impl reference`): the C++
restatement of ParallelHashAggregate (exec/parallel.go:109-314) timed on the
host cores over the benchmark's workload, printing one JSON line with the
same metric, unit, direction and config as the GPU arm, plus `impl`,
`cpu_baseline` and a zero-copy `e2e`. Under torchrun only rank 0 prints."""
from __future__ import annotations

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, env=e,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return [json.loads(ln) for ln in out.stdout.splitlines() if ln.startswith("{")]


def test_reference_arm_line():
    lines = run_bench("--impl", "reference", "--steps", "2", "--warmup", "3")
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["metric"] == "GB/s scanned" and d["unit"] == "GB/s"
    assert d["higher_is_better"] is True and d["steps"] == 2 and d["value"] > 0
    assert d["config"]["rows_per_gpu"] == 6_000_000 and d["config"]["bytes_per_step_per_gpu"] == 72 * 6_000_000
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_print_nothing():
    lines = run_bench("--impl", "reference", "--steps", "1", "--warmup", "3",
                      env={"WORLD_SIZE": "2", "RANK": "1", "LOCAL_RANK": "1"})
    assert lines == []
