"""bench.py's multi-process path on the CPU: two gloo ranks on 127.0.0.1.

The path does not shard (replicas only): every rank runs its own problem, the step time is the
maximum over ranks, and the reference arm runs on rank 0 alone.  These tests run the same code
with world size 2 over gloo, without a GPU.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


WORKER = r"""
import datetime, json, os, sys
sys.path.insert(0, os.environ["ROOT"])
import torch.distributed as dist
import bench
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
rank = dist.get_rank()
# the slowest rank's time is the job's time
ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist)
# replicas draw different problems (seed 1 + 10 rank)
a = bench.phi_matrix(4, 3, 1.0, 1 + 10 * rank)
vals = [None, None]
dist.all_gather_object(vals, float(a.sum()))
print(json.dumps({"rank": rank, "ms": ms, "distinct": vals[0] != vals[1]}))
dist.barrier()
dist.destroy_process_group()
"""


def _launch(code, nproc=2, extra_args=()):
    port = _free_port()
    procs = []
    for r in range(nproc):
        env = dict(os.environ, ROOT=ROOT, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(nproc),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", code, *extra_args], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=120)
        except subprocess.TimeoutExpired:
            p.kill()
            raise
        assert p.returncode == 0, e[-2000:]
        outs.append(o)
    return outs


def test_step_time_is_max_over_two_gloo_ranks():
    outs = _launch(WORKER)
    rows = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert sorted(r["rank"] for r in rows) == [0, 1]
    assert all(r["ms"] == 15.0 for r in rows), rows
    assert all(r["distinct"] for r in rows), rows


REF_ARM = r"""
import os, sys
sys.path.insert(0, os.environ["ROOT"])
import bench
class A:
    gpus, steps, warmup, ref_rows = 2, 1, 0, 2
rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
if rank != 0:
    sys.exit(bench.run_reference_arm(A, rank, world))
print("rank0")
"""


def test_reference_arm_other_ranks_exit_without_work():
    """Under torchrun the reference arm runs on rank 0 only; rank 1 returns 0 and prints nothing."""
    outs = _launch(REF_ARM)
    assert outs[0].strip() == "rank0"
    assert outs[1].strip() == ""
