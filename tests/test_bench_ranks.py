"""bench.py's host logic: the schedule, the PM byte count, and the multi-GPU side with two ranks
over gloo on CPU (127.0.0.1).

A run on N GPUs is N independent replicas (no data-path collective): each rank advances its own
particles, the job's time is the slowest rank's, and the whole-job rate counts every rank's
particles. The reference arm runs on rank 0 only; the other ranks return without work."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

RANK_SCRIPT = r"""
import json, os, sys
from datetime import timedelta
import torch
import torch.distributed as dist
sys.path.insert(0, sys.argv[1])
import bench
rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", timeout=timedelta(seconds=30))
ms_local = 10.0 + 5.0 * rank
dist.barrier()
ms = bench.max_over_ranks(ms_local, dist, torch.device("cpu"))
ref = bench.run_reference(None, rank, world) if rank != 0 else "skipped"
out = {"rank": rank, "ms": ms, "seed": bench.replica_seed(7, rank),
       "rate": bench.job_rate(1000, world, 4, ms), "ref_is_none": ref is None}
dist.barrier()
dist.destroy_process_group()
print(json.dumps(out), flush=True)
"""


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_gloo():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                   WORLD_SIZE="2", LOCAL_RANK=str(rank))
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_SCRIPT, str(ROOT)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            so, se = p.communicate(timeout=120)
        finally:
            if p.poll() is None:
                p.kill()
        assert p.returncode == 0, se[-2000:]
        outs.append(json.loads(so.strip().splitlines()[-1]))
    outs.sort(key=lambda d: d["rank"])
    # the slowest rank's time on every rank, so that both compute the same line
    assert outs[0]["ms"] == outs[1]["ms"] == 15.0
    # replicas differ in their seeds only
    assert outs[0]["seed"] != outs[1]["seed"]
    # whole-job throughput: both ranks' particles over the slowest rank's time
    assert outs[0]["rate"] == outs[1]["rate"] == 1000 * 2 * 4 / 0.015
    # the reference arm does no work off rank 0
    assert outs[1]["ref_is_none"]


def test_schedule_and_pm_bytes():
    """The step schedule is uniform in ln a from the initial a and reaches a = 1 on its last step
    (runner.rs:240); the PM byte count is the documented 36N + 64M."""
    import math
    sys.path.insert(0, str(ROOT))
    import bench
    a = bench.schedule(128, 128)
    assert len(a) == 128 and abs(a[-1] - 1.0) < 1e-6
    r = [math.log(a[i + 1] / a[i]) for i in range(len(a) - 1)]
    assert max(r) - min(r) < 1e-5
    assert a[0] > bench.A_INIT
    assert bench.pm_bytes_per_step(256 ** 3, 512) == 36 * 256 ** 3 + 64 * 512 ** 3
