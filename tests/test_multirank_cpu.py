"""Multi-GPU host logic on CPU: replica sharding (longest-processing-time
balance by atom count) and the max/sum-over-ranks reductions, run as two
gloo ranks on 127.0.0.1; the bench's reference arm under torchrun (rank 0
reports, other ranks exit without work)."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_lpt_partition_balances_replicas():
    from tdmd_claude_b200 import workloads as W
    from tdmd_claude_b200.replicas import lpt_partition
    sizes = [s.n for s in W.replica_set(64, seed=5)]
    for parts in (1, 2, 3, 8):
        bins = lpt_partition(sizes, parts)
        flat = sorted(i for b in bins for i in b)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in b) for b in bins]
        # LPT: the heaviest bin exceeds the mean by at most the largest item
        assert max(loads) - np.mean(loads) <= max(sizes)
    assert lpt_partition([5, 3, 2], 2) == [[0], [1, 2]]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    from tdmd_claude_b200.replicas import max_over_ranks, sum_over_ranks
    mx = max_over_ranks(1.5 + rank, dist)
    sm = sum_over_ranks(10 * (rank + 1), dist)
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump({"max": mx, "sum": sm}, f)


def test_reductions_over_two_gloo_ranks(tmp_path):
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    for r in range(2):
        got = json.load(open(tmp_path / f"r{r}.json"))
        assert got == {"max": 2.5, "sum": 30.0}


def test_reference_arm_under_torchrun_env(tmp_path):
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--gpus", "2", "--steps", "1", "--warmup", "3"],
                         capture_output=True, text=True, timeout=300, env=env)
    assert out.returncode == 0 and out.stdout.strip() == ""


def test_reference_arm_prints_its_line():
    """bench.py --impl reference on rank 0: one JSON line with the arm's
    contract keys (the reference CPU loop, a bounded sample)."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "3"],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "atom-steps/s" and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
