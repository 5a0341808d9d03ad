"""CPU: the multi-rank plumbing of bench.py with world size 2 over gloo.

bench.py --gpus N runs N independent replicas of the step (the path does not
shard; no collective is on the data path) and reports the job's time as the
maximum over ranks.  Here two CPU processes check that reduction and that the
reference arm lets every rank but 0 exit without work.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import os, sys, json
sys.path.insert(0, sys.argv[1])
import torch.distributed as dist
import bench
dist.init_process_group("gloo", init_method="env://")
rank = dist.get_rank()
got = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 3.5], dist, "cpu")
# the reference arm: ranks other than 0 return 0 without printing
args = bench._args(["--impl", "reference", "--gpus", "2"])
rc = bench.run_reference(args) if rank != 0 else 0
print(json.dumps({"rank": rank, "max": got, "ref_rc": rc}), flush=True)
dist.destroy_process_group()
"""


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_bench_max_over_ranks_gloo_world_2(tmp_path):
    script = tmp_path / "worker.py"
    script.write_text(WORKER)
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, str(script), ROOT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    for o in outs:
        assert o["max"] == [2.0, 10.0, 3.5]
        assert o["ref_rc"] == 0
