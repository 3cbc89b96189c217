"""Multi-rank plumbing of bench.py on CPU with the gloo backend (world size
2, no GPU): the slowest rank's time and the whole-job rate, and the
reference arm under torchrun (rank 0 alone prints its line, the other rank
exits 0 without work). The GPU path itself is replicas only: one process per
GPU with no data-path collective."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, queue):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    local = 1.5 + rank  # rank 1 is the slower one
    slowest = bench.max_over_ranks(local, dist, "cpu")
    queue.put((rank, slowest, bench.replica_rate(world, 1000, 4, slowest)))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_rate_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(queue.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in results] == [2.5, 2.5]
    assert results[0][2] == pytest.approx(2 * 1000 * 4 / 2.5)


def test_reference_arm_under_torchrun():
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"), "--impl",
           "reference", "--gpus", "2", "--steps", "1", "--warmup", "3", "--cpu-scale", "4", "--cpu-workers", "2"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=str(ROOT))
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["value"] > 0 and line["n_gpus"] == 2
    assert line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["h2d_bytes_per_step"] == 0
