"""Helpers for the slab-decomposition tests: run an application on R ranks
(one process each, gloo host transport, apps/run_dist.py) and put the
per-rank dumps back together along the slowest axis."""

from __future__ import annotations

import os
import socket
import subprocess
import sys

import numpy as np

from tests.opsdump import read_dump

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(name, flavour, args, ranks, dump, timeout=600, env=None):
    """Returns rank 0's stdout; every rank must exit 0."""
    port = free_port()
    procs = []
    for r in range(ranks):
        e = dict(os.environ, RANK=str(r), WORLD_SIZE=str(ranks), LOCAL_RANK="0",
                 MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), OPS_DUMP_FILE=dump,
                 PYTHONPATH=ROOT, **(env or {}))
        procs.append(subprocess.Popen([sys.executable, "-m", "apps.run_dist", name, flavour, *args],
                                      cwd=ROOT, env=e, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            o, err = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        outs.append((p.returncode, o, err))
    for r, (rc, o, err) in enumerate(outs):
        assert rc == 0, "rank %d failed (rc %d):\n%s\n%s" % (r, rc, o[-2000:], err[-3000:])
    return outs[0][1]


def gather(dump, ranks):
    """name -> flat array of the whole dat, the ranks' owned rows in order
    (rows along the slowest axis are the outermost in memory)."""
    parts = [read_dump("%s.r%d" % (dump, r)) for r in range(ranks)]
    out = {}
    for name, (meta, arr) in parts[0].items():
        pieces = [arr] + [p[name][1] for p in parts[1:] if name in p]
        out[name] = (meta, np.concatenate(pieces))
    return out
