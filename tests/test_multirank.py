"""The multi-rank side of bench.py, on CPU: two gloo ranks as child processes.

`bench.py --gpus N` runs one replica per rank (the path does not shard) and
reports the whole-job value over the slowest rank's time. These tests cover
that host logic without a GPU: the max-over-ranks reduction, the whole-job
aggregate, and the reference arm, which does its work on rank 0 alone."""
import argparse
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

RANK_CODE = r"""
import datetime, json, os, sys
sys.path.insert(0, os.environ["AEFDTD_ROOT"])
import torch.distributed as dist
import bench
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=30))
ws, rank, _ = bench.dist_env()
mine = 10.0 + 5.0 * rank
ms = bench.max_over_ranks(mine, device="cpu")
value = bench.whole_job_gcells(1000000, 640, ms, ws)
dist.barrier()
dist.destroy_process_group()
print(json.dumps({"rank": rank, "ws": ws, "mine": mine, "ms": ms, "value": value}))
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_take_the_slowest_time_and_sum_the_replicas():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), AEFDTD_ROOT=ROOT)
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_CODE], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err[-2000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    assert sorted(o["rank"] for o in outs) == [0, 1]
    for o in outs:
        assert o["ws"] == 2
        assert o["ms"] == 15.0          # rank 1's 15 ms, the slower replica
        # two replicas of 1e6 cells x 640 steps over 15 ms
        assert abs(o["value"] - 2 * 1e6 * 640 / 15e-3 / 1e9) < 1e-9


def test_without_a_group_the_time_is_returned_as_given():
    assert bench.max_over_ranks(12.5, device="cpu") == 12.5
    assert abs(bench.whole_job_gcells(2000000, 64, 4.0, 1) - 2e6 * 64 / 4e-3 / 1e9) < 1e-9


def test_reference_arm_does_no_work_on_other_ranks(monkeypatch, capsys):
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("LOCAL_RANK", "1")
    args = argparse.Namespace(gpus=2, steps=3, warmup=3, impl="reference")
    assert bench.reference_arm(args) is None
    assert capsys.readouterr().out == ""
