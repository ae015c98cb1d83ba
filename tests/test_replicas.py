"""The benchmark's multi-process path on CPU: two gloo ranks, as torchrun
launches them, align on barriers, agree on the maximum of their times, and
only rank 0 reports; the reference arm runs on rank 0 alone."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import json, os, sys, time
sys.path.insert(0, {root!r})
from minimumlbvh_b200.replicas import Replicas
r = Replicas("gloo", timeout_s=60)
r.barrier()
mine = 1.0 + r.rank  # each rank's own "time"
out = {{"rank": r.rank, "world": r.world, "max": r.max(mine), "root": r.is_root}}
r.barrier()
r.close()
print(json.dumps(out), flush=True)
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _launch(code, world):
    port = _free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=120)
        assert p.returncode == 0, e[-2000:]
        outs.append(o)
    return outs


def test_two_gloo_ranks_agree_on_max_and_root():
    outs = _launch(WORKER.format(root=ROOT), 2)
    res = sorted((json.loads(o.strip().splitlines()[-1]) for o in outs), key=lambda d: d["rank"])
    assert [d["world"] for d in res] == [2, 2]
    assert [d["max"] for d in res] == [2.0, 2.0]
    assert [d["root"] for d in res] == [True, False]


def test_single_process_is_a_no_op():
    from minimumlbvh_b200.replicas import Replicas
    env = {k: os.environ.pop(k) for k in ("RANK", "WORLD_SIZE") if k in os.environ}
    try:
        r = Replicas("gloo")
        r.barrier()
        assert r.max(3.5) == 3.5 and r.is_root and r.world == 1
        r.close()
    finally:
        os.environ.update(env)


def test_reference_arm_runs_on_rank_zero_only(tmp_path):
    """bench.py --impl reference under two ranks: rank 1 exits 0 without work
    or output (rank 0 would time the reference CPU code; it is skipped here by
    running rank 1 alone)."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""
