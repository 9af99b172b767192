"""The replicas path of bench.py on two gloo ranks (CPU): the whole-job time is the slowest
rank's and the simulated days of all replicas add up; the reference arm prints only on rank 0."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import os, sys, json, datetime
sys.path.insert(0, sys.argv[1])
import torch.distributed as dist
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
import bench
rank = dist.get_rank()
ms, days = bench.reduce_over_ranks(10.0 + 5.0 * rank, 1.5 + rank, dist.get_world_size(), device="cpu")
print(json.dumps({"rank": rank, "ms": ms, "days": days}), flush=True)
dist.barrier()
dist.destroy_process_group()
"""


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_reduce_over_ranks_two_gloo_ranks(tmp_path):
    script = tmp_path / "worker.py"
    script.write_text(WORKER)
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, str(script), ROOT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    for o in outs:
        assert o["ms"] == 15.0          # the slower rank
        assert o["days"] == 1.5 + 2.5   # all replicas' simulated days


def test_reference_arm_prints_only_on_rank0(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = bench.argparse.Namespace(workload="strat1024x8", warmup=1, steps=1)
    bench.reference_arm(args)
    assert capsys.readouterr().out == ""
