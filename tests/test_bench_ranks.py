"""The multi-rank side of bench.py on the CPU: two gloo ranks run the same
combination the GPU ranks run over NCCL (replicas, max over ranks of the device
time and of the end-to-end time, whole-job throughput)."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import json, os, sys
sys.path.insert(0, sys.argv[1])
import torch.distributed as dist
import bench
dist.init_process_group("gloo")
rank, world = dist.get_rank(), dist.get_world_size()
out = bench.aggregate(dist, "cpu", ms_step=0.25 * (rank + 1), e2e_s=1.0 + rank, n=1000, steps=10, world=world)
print(json.dumps(out))
dist.barrier()
dist.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_take_the_slowest_rank():
    import json

    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2",
                   LOCAL_RANK=str(rank))
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER, ROOT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=120)
        except subprocess.TimeoutExpired:
            p.kill()
            pytest.fail("gloo rank did not finish")
        assert p.returncode == 0, e
        outs.append(json.loads(o.strip().splitlines()[-1]))
    for o in outs:
        assert o["ms_step"] == pytest.approx(0.5)           # the slower rank
        assert o["value"] == pytest.approx(2 * 1000 / 0.5e-3)
        assert o["e2e_rate"] == pytest.approx(2 * 1000 * 10 / 2.0)


def test_single_rank_needs_no_collective():
    sys.path.insert(0, ROOT)
    import bench

    o = bench.aggregate(None, "cpu", ms_step=0.5, e2e_s=2.0, n=1000, steps=10, world=1)
    assert o["value"] == pytest.approx(1000 / 0.5e-3) and o["e2e_rate"] == pytest.approx(5000.0)
