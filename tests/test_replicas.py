"""The replicas path for more than one GPU, run as two gloo ranks on CPU: the max over
ranks of a timing, the sum of frame counts, the barrier, and distinct frames per replica.
No data-path collective exists; these are all the collectives bench.py takes."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, os, sys, time
sys.path.insert(0, os.environ["GB_ROOT"])
from libgail_b200.replicas import Replicas
r = Replicas(backend="gloo", timeout_s=30)
t = 1.5 * (r.rank + 1)          # this rank's "elapsed time"
r.barrier()
out = {"rank": r.rank, "world": r.world, "max": r.max(t), "sum": r.sum(48), "seed": r.frame_seed(1000)}
r.barrier()
r.close()
print(json.dumps(out))
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(world):
    port = _free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), GB_ROOT=ROOT, CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=120)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        assert p.returncode == 0, e
        outs.append(json.loads(o.strip().splitlines()[-1]))
    return sorted(outs, key=lambda d: d["rank"])


def test_two_replicas_gloo():
    outs = _run(2)
    assert [o["rank"] for o in outs] == [0, 1]
    assert all(o["world"] == 2 for o in outs)
    assert all(o["max"] == 3.0 for o in outs)       # max over ranks of 1.5, 3.0
    assert all(o["sum"] == 96.0 for o in outs)      # whole-job frames: 2 x 48
    assert outs[0]["seed"] != outs[1]["seed"]       # each replica its own frames


def test_one_replica_needs_no_group():
    from libgail_b200.replicas import Replicas
    old = {k: os.environ.pop(k, None) for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE")}
    try:
        r = Replicas(backend="gloo")
        assert (r.rank, r.world) == (0, 1)
        assert r.max(2.5) == 2.5 and r.sum(7) == 7.0
        r.barrier()
        r.close()
    finally:
        for k, v in old.items():
            if v is not None:
                os.environ[k] = v


@pytest.mark.parametrize("world", [3])
def test_more_replicas_gloo(world):
    outs = _run(world)
    assert all(o["max"] == 1.5 * world for o in outs)
    assert len({o["seed"] for o in outs}) == world
