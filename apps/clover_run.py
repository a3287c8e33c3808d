"""Run the CloverLeaf step harness (apps/clover_step) in one flavour.

    python -m apps.clover_run --flavour b200|oracle|ref_omp|ref_cuda --cells N --steps K
                              [--warmup W] [--seed S] [--dump FILE] [--fetch-dump FILE]
                              [--threads T]

Writes the input deck of the 2D hydro configuration into a scratch directory
(background rho=0.2 e=1.0 on a 10x10 domain, a cell-aligned 2.5x2.5 square of
rho=1.0 e=2.5 whose position is drawn from the seed), runs W untimed and K
timed steps through the harness's C entry points, and prints one JSON line:
the field summary of the final state (volume, mass, pressure, internal and
kinetic energy), the per-step time and the steps run.  The field summary is
taken after the timed steps, outside the timed region.

--dump writes every live dat with halos at ops_exit (this backend and the
oracle only); --fetch-dump writes every dat's interior through
ops_dat_fetch_data (clover_step_dump), which works on every flavour, the
reference's OpenMP backend included.

Each flavour runs in its own process (every flavour exports the same OPS
symbols).
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import random
import re
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def make_deck(cells: int, seed: int, end_step: int = 1000000) -> str:
    """Deck of the hydro configuration; the high-density square covers 1/16
    of the 10x10 domain at a seeded, cell-aligned position."""
    rng = random.Random(seed)
    dx = 10.0 / cells
    side = cells // 4  # 2.5 / 10 of the cells
    i0 = rng.randrange(0, cells - side + 1)
    j0 = rng.randrange(0, cells - side + 1)
    x0, y0 = i0 * dx, j0 * dx
    x1, y1 = (i0 + side) * dx, (j0 + side) * dx
    return ("*clover\n"
            " state 1 density=0.2 energy=1.0\n"
            " state 2 density=1.0 energy=2.5 geometry=rectangle "
            "xmin=%.15f xmax=%.15f ymin=%.15f ymax=%.15f\n"
            " x_cells=%d\n y_cells=%d\n"
            " xmin=0.0\n ymin=0.0\n xmax=10.0\n ymax=10.0\n"
            " initial_timestep=0.04\n timestep_rise=1.5\n max_timestep=0.04\n"
            " end_time=1000.0\n end_step=%d\n"
            "*endclover\n" % (x0, x1, y0, y1, cells, cells, end_step))


def parse_summary(text: str):
    """Last field-summary line of clover.out: step, vol, mass, density,
    pressure, ie, ke, total."""
    rows = re.findall(r"step:\s+(\d+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)",
                      text)
    if not rows:
        return None
    r = rows[-1]
    keys = ["step", "volume", "mass", "density", "pressure", "ie", "ke", "total"]
    return {k: (int(v) if k == "step" else float(v)) for k, v in zip(keys, r)}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--flavour", required=True)
    ap.add_argument("--cells", type=int, default=240)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=0)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--dump", default=None)
    ap.add_argument("--fetch-dump", default=None)
    ap.add_argument("--threads", type=int, default=0)
    a = ap.parse_args(argv)
    from apps.catalog import artifact
    lib = artifact("clover_step", a.flavour, shared=True)
    if not os.path.exists(lib):
        raise SystemExit("not built: %s" % lib)
    if a.threads:
        os.environ["OMP_NUM_THREADS"] = str(a.threads)
    if a.dump:
        os.environ["OPS_DUMP_FILE"] = os.path.abspath(a.dump)
    if a.fetch_dump:
        a.fetch_dump = os.path.abspath(a.fetch_dump)
    work = tempfile.mkdtemp(prefix="clover_")
    with open(os.path.join(work, "clover.in"), "w") as f:
        f.write(make_deck(a.cells, a.seed))
    os.chdir(work)
    L = ctypes.CDLL(lib, mode=ctypes.RTLD_GLOBAL)
    L.clover_step_run.restype = ctypes.c_double
    argv_c = (ctypes.c_char_p * 2)(b"clover_step", None)
    L.clover_step_setup(1, argv_c)
    if a.warmup:
        L.clover_step_run(a.warmup)
    L.clover_step_sync()
    t0 = time.perf_counter()
    L.clover_step_run(a.steps)
    L.clover_step_sync()
    t1 = time.perf_counter()
    L.clover_step_summary()
    if a.fetch_dump:
        L.clover_step_dump.argtypes = [ctypes.c_char_p]
        if L.clover_step_dump(a.fetch_dump.encode()) != 0:
            raise SystemExit("clover_step_dump failed")
    L.clover_step_finish()
    summ = parse_summary(open(os.path.join(work, "clover.out")).read())
    print(json.dumps({"flavour": a.flavour, "cells": a.cells, "steps": a.steps,
                      "warmup": a.warmup, "s_per_step": (t1 - t0) / max(a.steps, 1),
                      "summary": summ, "workdir": work}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
