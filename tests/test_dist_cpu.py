"""The N>1 plumbing of bench.py (one process per GPU, replicas, max-over-ranks
timing) on CPU: two gloo ranks on 127.0.0.1."""

import os
import socket
import subprocess
import sys

import numpy as np
import pytest

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


# ---------------------------------------------------------------------------
# slab decomposition (include/ops_b200_dist.h) on the CPU oracle: the same
# program on 2 and 3 gloo ranks gives every dat bit for bit as on one rank
# ---------------------------------------------------------------------------
def _oracle_poisson_dist(tmp_path, ranks, args):
    from tests.apprun import ensure, result_lines, run_app
    from tests.distrun import gather, run_ranks
    from tests.opsdump import read_dump
    ensure("poisson_mb", "oracle")
    one_out, one_dump = run_app("poisson_mb", "oracle", args, dump=True)
    dump = str(tmp_path / "dist.dump")
    out = run_ranks("poisson_mb", "oracle", args, ranks, dump)
    whole = read_dump(one_dump)
    parts = gather(dump, ranks)
    assert set(parts) == set(whole)
    for name, (meta, arr) in whole.items():
        assert np.array_equal(parts[name][1], arr), name
    # max-residual reductions are exact; the checksum sums in another order
    res = lambda t: [l for l in result_lines(t, ("sweep",))]
    assert res(out) == res(one_out) and res(out)
    c1 = float([l for l in result_lines(out, ("checksum",))][0].split()[1])
    c0 = float([l for l in result_lines(one_out, ("checksum",))][0].split()[1])
    assert abs(c1 - c0) <= 1e-13 * abs(c0)


@pytest.mark.parametrize("ranks,args", [(2, ["-nb=1", "-n=64", "-sweeps=30", "-check=10"]),
                                        (3, ["-nb=1", "-n=61", "-sweeps=25", "-check=5"])])
def test_oracle_slab_decomposition_matches_one_rank(tmp_path, ranks, args):
    _oracle_poisson_dist(tmp_path, ranks, args)


def test_slab_partition_arithmetic():
    """the shared decomposition arithmetic: slabs tile [0, G) and differ by
    at most one row; clipping keeps the global halo rows on the end ranks"""
    import ctypes
    for G in (7, 64, 1000):
        for R in (1, 2, 3, 8):
            if R > G:
                continue
            b = [(G * r // R, G * (r + 1) // R) for r in range(R)]
            assert b[0][0] == 0 and b[-1][1] == G
            assert all(b[i][1] == b[i + 1][0] for i in range(R - 1))
            assert max(h - l for l, h in b) - min(h - l for l, h in b) <= 1
