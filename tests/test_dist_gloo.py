"""bench.py's N > 1 plumbing on the CPU: two gloo ranks.

With N GPUs the bench runs one process per GPU, each solving its own replica
of the problem (the path has no exchange between problems); the only
collectives are the barrier around a timed region and the max of the
per-rank times, and the reported rate is the whole job's.  Here the same
`Ranks` object runs with the gloo backend on two CPU processes, and the
reference arm is checked to do nothing on ranks other than 0.
"""
import json
import os
import socket
import subprocess
import sys
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import json, os, sys
sys.path.insert(0, os.environ["BENCH_ROOT"])
import torch
import bench
rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
r = bench.Ranks(world, "gloo", torch.device("cpu"), timeout_s=60)
r.barrier()
m = r.max(1.0 + rank)                 # a per-rank time
rate = r.total_rate(10, 2.0 + rank)   # 10 units on every rank
r.barrier()
r.close()
print(json.dumps({"rank": rank, "max": m, "rate": rate}), flush=True)
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_time_and_rate():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2",
                   LOCAL_RANK=str(rank), BENCH_ROOT=ROOT)
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err[-2000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    assert sorted(o["rank"] for o in outs) == [0, 1]
    for o in outs:
        assert o["max"] == 2.0                      # the slower rank's time, on both ranks
        assert o["rate"] == pytest.approx(2 * 10 / 3.0)  # whole job: 2 ranks x 10 units / max time


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import torch
    import bench
    r = bench.Ranks(1, "gloo", torch.device("cpu"))
    assert r.pg is None
    assert r.max(3.5) == 3.5
    assert r.total_rate(7, 2.0) == pytest.approx(3.5)
    r.barrier()
    r.close()


def test_reference_arm_is_rank_zero_only(capsys):
    sys.path.insert(0, ROOT)
    import bench
    args = types.SimpleNamespace(config=2, scale=1.0, steps=1, warmup=0)
    assert bench.run_reference(args, 1, 2) is None
    assert capsys.readouterr().out == ""
