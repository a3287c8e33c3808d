"""The N>1 plumbing of bench.py (one process per GPU, replicas, max-over-ranks
timing) on CPU: two gloo ranks on 127.0.0.1."""

import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import os, sys, json
sys.path.insert(0, %r)
import bench
d = bench.Dist()
d.barrier()
mx = d.max(float(d.rank + 1) * 1.5)
sm = d.sum(float(d.rank + 1))
d.barrier()
print(json.dumps({"rank": d.rank, "world": d.world, "max": mx, "sum": sm}))
d.close()
"""


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_max_and_sum():
    import json
    port = free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD % ROOT], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=120) for p in procs]
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e[-2000:]
    res = [json.loads([l for l in o.splitlines() if l.startswith("{")][-1]) for o, _ in outs]
    for r in res:
        assert r["world"] == 2 and r["max"] == 3.0 and r["sum"] == 3.0
