"""The multi-rank side of bench.py on CPU: two gloo ranks (one process each, rendezvous on
127.0.0.1) agree on the whole-job time as the maximum of their own times, the job value counts
every rank's replica, and the reference arm runs on rank 0 alone."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r"""
import datetime, json, os, sys
sys.path.insert(0, os.environ["AMX_ROOT"])
import torch.distributed as dist
import bench
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
rank = dist.get_rank()
local = [3.25, 7.5][rank]
t = bench.job_time_ms(local, dist, "cpu")
print(json.dumps({"rank": rank, "job_ms": t, "value": bench.job_value(dist.get_world_size(), 1e9, t)}))
dist.barrier()
dist.destroy_process_group()
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_take_the_max_time():
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2",
                   LOCAL_RANK=str(rank), AMX_ROOT=ROOT)
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_SCRIPT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err[-2000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    assert sorted(o["rank"] for o in outs) == [0, 1]
    for o in outs:
        assert o["job_ms"] == 7.5
        assert o["value"] == pytest.approx(2 * 1e9 / 7.5e-3 / 1e9)


def test_single_rank_time_and_value():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.job_time_ms(4.0) == 4.0
    assert bench.job_value(1, 2e9, 1.0) == pytest.approx(2000.0)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
