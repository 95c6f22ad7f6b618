"""Multi-process host logic of bench.py on CPU (gloo, world size 2).

The solve path does not shard (one replica per GPU), so the only cross-rank
steps are the barrier around the timed region, the max over ranks of the
measured time, and rank 0 alone printing the JSON line.  These run here with
the gloo backend; no GPU is used.
"""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    import bench
    w, r, _ = bench.dist_setup("gloo")
    assert (w, r) == (world, rank)
    bench.barrier(w)
    # each rank reports a different time; every rank must see the largest
    got = bench.max_over_ranks(1.5 * (rank + 1), w)
    assert got == 1.5 * world, got
    bench.barrier(w)
    dist.destroy_process_group()


def test_max_over_ranks_and_barrier_gloo():
    import torch.multiprocessing as mp
    mp.spawn(_rank_main, args=(2, _free_port()), nprocs=2, join=True)


def test_reference_arm_prints_once_under_torchrun():
    # side 16 has no measured reference iteration count, so rank 0 reports an
    # `unavailable` line after its quick sample; rank 1 must print nothing
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           str(ROOT / "bench.py"), "--impl", "reference", "--side", "16", "--dist-backend", "gloo"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    assert lines[0]["impl"] == "reference"
