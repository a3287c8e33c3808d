"""Helpers for tests: build and run application flavours, parse their output.

The b200 and oracle flavours run as shared libraries loaded by a child Python
process (apps/run_shared.py), so the backend library is loaded by a Python
process; each run is its own process because OPS state is process-global.
"""

from __future__ import annotations

import os
import re
import subprocess
import sys
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def ensure(name: str, flavour: str, shared: bool = True) -> str:
    from apps import catalog
    path = catalog.artifact(name, flavour, shared)
    if os.path.exists(path):
        return path
    if not catalog.available(name):
        pytest.skip("%s/%s not built and its sources are not present" % (name, flavour))
    return catalog.build(name, flavour, shared=shared)


def run_app(name: str, flavour: str, args=(), dump: bool = False, cwd=None, timeout=900,
            env=None):
    """Returns (stdout, dump_path or None).  env: extra environment variables."""
    ensure(name, flavour, shared=True)
    env = dict(os.environ, **(env or {}))
    dpath = None
    if dump:
        fd, dpath = tempfile.mkstemp(prefix="%s_%s_" % (name, flavour), suffix=".dump")
        os.close(fd)
        env["OPS_DUMP_FILE"] = dpath
    r = subprocess.run([sys.executable, "-m", "apps.run_shared", name, flavour, *args],
                       cwd=cwd or ROOT, env=dict(env, PYTHONPATH=ROOT), capture_output=True,
                       text=True, timeout=timeout)
    if r.returncode != 0:
        raise AssertionError("%s/%s failed (rc %d):\n%s\n%s" % (name, flavour, r.returncode,
                                                                 r.stdout[-3000:], r.stderr[-3000:]))
    return r.stdout, dpath


def run_exe(name: str, flavour: str, args=(), cwd=None, timeout=900):
    exe = ensure(name, flavour, shared=False)
    r = subprocess.run([exe, *args], cwd=cwd, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise AssertionError("%s/%s failed (rc %d):\n%s" % (name, flavour, r.returncode,
                                                             r.stderr[-3000:]))
    return r.stdout


def result_lines(text: str, keys=("sweep", "checksum", "sums", "min", "max", "count",
                                  "fetch_b", "fp64", "fp32")):
    return [l for l in text.splitlines() if l.split() and l.split()[0] in keys]


def floats(line: str):
    return [float(x) for x in re.findall(r"-?\d+\.\d+(?:e[-+]\d+)?|-?\d+e[-+]\d+", line)]


def assert_lines_close(got, want, rtol):
    assert len(got) == len(want), (got, want)
    for g, w in zip(got, want):
        assert g.split()[0] == w.split()[0], (g, w)
        fg, fw = floats(g), floats(w)
        assert len(fg) == len(fw), (g, w)
        for a, b in zip(fg, fw):
            assert abs(a - b) <= rtol * max(abs(b), 1e-300), (g, w, abs(a - b) / max(abs(b), 1e-300))


def clover_deck_test1() -> str:
    """CloverLeaf test problem 1 (the reference's default deck parameters,
    field_summary.cpp:91): 10 x 2 cells on a 10 x 2 domain, a dense region
    over x in [0,5], run to t = 3.0."""
    return ("*clover\n state 1 density=0.2 energy=1.0\n"
            " state 2 density=1.0 energy=2.5 geometry=rectangle xmin=0.0 xmax=5.0 ymin=0.0 "
            "ymax=2.0\n x_cells=10\n y_cells=2\n xmin=0.0\n ymin=0.0\n xmax=10.0\n ymax=2.0\n"
            " initial_timestep=0.04\n timestep_rise=1.5\n max_timestep=0.04\n end_time=3.0\n"
            " test_problem 1\n*endclover\n")


def clover_deck_test2() -> str:
    """CloverLeaf test problem 2 (field_summary.cpp:92): 960 x 960 cells on a
    10 x 10 domain, 87 steps."""
    return ("*clover\n state 1 density=0.2 energy=1.0\n"
            " state 2 density=1.0 energy=2.5 geometry=rectangle xmin=0.0 xmax=5.0 ymin=0.0 "
            "ymax=2.0\n x_cells=960\n y_cells=960\n xmin=0.0\n ymin=0.0\n xmax=10.0\n ymax=10.0\n"
            " initial_timestep=0.04\n timestep_rise=1.5\n max_timestep=0.04\n end_step=87\n"
            " test_problem 2\n*endclover\n")


def clover3d_deck_test2() -> str:
    """CloverLeaf 3D test problem 2 (CloverLeaf_3D/field_summary.cpp:95,
    expected kinetic energy 20.0546870878964): 96^3 cells on a 10^3 domain, a
    dense cuboid [0,5] x [0,2] x [0,4], 87 steps.  checkpoint_frequency must be
    set: the app takes `step % checkpoint_frequency` every step
    (CloverLeaf_3D/clover_leaf.cpp:209) and gives it no default."""
    return ("*clover\n state 1 density=0.2 energy=1.0\n"
            " state 2 density=1.0 energy=2.5 geometry=cuboid xmin=0.0 xmax=5.0 ymin=0.0 "
            "ymax=2.0 zmin=0.0 zmax=4.0\n x_cells=96\n y_cells=96\n z_cells=96\n"
            " xmin=0.0\n ymin=0.0\n zmin=0.0\n xmax=10.0\n ymax=10.0\n zmax=10.0\n"
            " initial_timestep=0.1\n max_timestep=0.1\n end_step=87\n end_time=1000.1\n"
            " test_problem 2\n checkpoint_frequency=10\n*endclover\n")


def tealeaf_deck_test1(solver: str = "tl_use_jacobi") -> str:
    """TeaLeaf test problem 1 (TeaLeaf/field_summary.cpp:84, expected
    temperature 157.55084183279294): 10 x 10 cells on a 10 x 10 domain, four
    low-density strips over a dense background, 10 steps, solver tolerance
    1e-15 (the reference's default deck uses Jacobi; CG and Chebyshev reach the
    same solution)."""
    states = [" state 1 density=100.0 energy=0.0001"]
    for k, (e, x0, x1, y0, y1) in enumerate([(25.0, 0, 1, 1, 2), (0.1, 1, 6, 1, 2),
                                              (0.1, 5, 6, 1, 8), (0.1, 5, 10, 7, 8)]):
        states.append(" state %d density=0.1 energy=%s geometry=rectangle xmin=%.1f xmax=%.1f "
                      "ymin=%.1f ymax=%.1f" % (k + 2, e, x0, x1, y0, y1))
    return ("*tea\n" + "\n".join(states) +
            "\n x_cells=10\n y_cells=10\n xmin=0.0\n ymin=0.0\n xmax=10.0\n ymax=10.0\n"
            " initial_timestep=0.004\n end_step=10\n tl_max_iters=1000\n %s\n tl_eps=1e-15\n"
            " test_problem 1\n*endtea\n" % solver)
