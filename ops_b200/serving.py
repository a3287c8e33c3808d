"""Solve serving on one B200: continuous batching of Poisson / heat / ADI requests.

    python -m ops_b200.serving [--requests 2000] [--rate R] [--mode mixed|fp64|both]
                               [--budget-gb 160] [--iters 16] [--seed 6] [--heat-frac F]

A request stream (seeded): Poisson-process arrivals; 70 % 2D Poisson solves
(5-point, zero Dirichlet boundary, n log-uniform in [64, 2048], f ~ U(-1,1),
relative residual 1e-8) and 30 % 3D ADI heat runs (n log-uniform in [32, 192],
u0 ~ U(-1,1), 10 steps); --heat-frac F turns a share F of the requests into
2D implicit heat runs (5 backward-Euler steps, each a CG solve to the same
tolerance, sizes as Poisson).  The serving loop keeps each admitted request's
arrays resident on the device and advances every active request in the same
batched launches (libops_b200.so, ob2s_*).  Admission: a request joins as
soon as it has arrived, a slot is free (OB2S_MAX_ACTIVE) and its bytes fit
the HBM budget; requests that arrive while others run join at the next
engine step.  Finished requests are retired at once.

Reported per mode: solves/s over the run, p50 / p99 latency (arrival to
completion, host clock), the bytes-model bandwidth, the worst final relative
residual, and for --mode both the FP64 one-request-at-a-time baseline on the
same stream and the relative difference of every mixed solution from its
FP64 counterpart.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import random
import sys
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "lib", "libops_b200.so")

POISSON2D, ADI3D, HEAT2D = 0, 1, 2
FP64, MIXED = 0, 1
MAX_ACTIVE = 128


class Result(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("n", ctypes.c_int), ("done", ctypes.c_int),
                ("iterations", ctypes.c_int), ("outer", ctypes.c_int),
                ("rel_residual", ctypes.c_double), ("checksum", ctypes.c_double)]


_lib = None


def lib():
    """libops_b200.so with the serving entry points typed; raises when the
    library or a CUDA device is missing (there is no CPU path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError("libops_b200.so is not built (make -C ops_b200)")
        L = ctypes.CDLL(LIB, mode=ctypes.RTLD_GLOBAL)
        vp, ip, i, d = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_double
        L.ob2s_create.argtypes = [ctypes.POINTER(vp), i, d, d, i, i]
        L.ob2s_destroy.argtypes = [vp]
        L.ob2s_destroy.restype = None
        L.ob2s_request_bytes.argtypes = [i, i, i]
        L.ob2s_request_bytes.restype = ctypes.c_size_t
        L.ob2s_submit.argtypes = [vp, i, i, i, i, ip]
        L.ob2s_run.argtypes = [vp, i, ip, i, ip]
        L.ob2s_active.argtypes = [vp]
        L.ob2s_result_of.argtypes = [vp, i, ctypes.POINTER(Result)]
        L.ob2s_fetch.argtypes = [vp, i, ctypes.POINTER(ctypes.c_double), ctypes.c_size_t]
        L.ob2s_release.argtypes = [vp, i]
        L.ob2s_reserve.argtypes = [vp, ctypes.c_size_t]
        L.ob2s_launches.argtypes = [vp]
        L.ob2s_launches.restype = ctypes.c_longlong
        L.ob2_error_string.argtypes = [i]
        L.ob2_error_string.restype = ctypes.c_char_p
        L.ob2_dev_init.argtypes = [i]
        _lib = L
    return _lib


def check(code: int, what: str) -> None:
    if code:
        msg = {200001: "no free request slot", 200002: "bad argument",
               200003: "request not finished"}.get(code)
        if msg is None:
            msg = lib().ob2_error_string(code).decode()
        raise RuntimeError("%s failed: %s (%d)" % (what, msg, code))


class Engine:
    """One serving engine (one precision mode) on the current device."""

    def __init__(self, mode: int, tol: float = 1e-8, inner_tol: float = 1e-2,
                 max_inner: int = 100000, tile_y: int = 32):
        L = lib()
        check(L.ob2_dev_init(int(os.environ.get("OPS_B200_DEVICE", "0"))), "device init")
        self.h = ctypes.c_void_p()
        check(L.ob2s_create(ctypes.byref(self.h), mode, tol, inner_tol, max_inner, tile_y),
              "ob2s_create")
        self.mode = mode
        self._ids = (ctypes.c_int * MAX_ACTIVE)()

    def close(self):
        if self.h:
            lib().ob2s_destroy(self.h)
            self.h = ctypes.c_void_p()

    def request_bytes(self, kind: int, n: int) -> int:
        return int(lib().ob2s_request_bytes(self.mode, kind, n))

    def submit(self, kind: int, n: int, seed: int, steps: int = 10) -> int:
        rid = ctypes.c_int()
        check(lib().ob2s_submit(self.h, kind, n, seed, steps, ctypes.byref(rid)), "ob2s_submit")
        return rid.value

    def run(self, iters: int) -> List[int]:
        nd = ctypes.c_int()
        check(lib().ob2s_run(self.h, iters, self._ids, MAX_ACTIVE, ctypes.byref(nd)), "ob2s_run")
        return [self._ids[k] for k in range(min(nd.value, MAX_ACTIVE))]

    def active(self) -> int:
        return lib().ob2s_active(self.h)

    def result(self, rid: int) -> Result:
        r = Result()
        check(lib().ob2s_result_of(self.h, rid, ctypes.byref(r)), "ob2s_result_of")
        return r

    def fetch(self, rid: int, count: int):
        import numpy as np
        out = np.empty(count, dtype=np.float64)
        check(lib().ob2s_fetch(self.h, rid, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                               count), "ob2s_fetch")
        return out

    def release(self, rid: int) -> None:
        check(lib().ob2s_release(self.h, rid), "ob2s_release")

    def launches(self) -> int:
        return int(lib().ob2s_launches(self.h))

    def reserve(self, nbytes: int) -> None:
        """Maps nbytes of device memory into the engine's pool once (server
        start-up), so that admitted requests reuse mapped memory."""
        check(lib().ob2s_reserve(self.h, nbytes), "ob2s_reserve")

    def reserve_up_to(self, nbytes: int) -> int:
        """reserve() of nbytes, or of the largest half-step below it that the
        device can hold; returns the bytes reserved."""
        while nbytes >= (1 << 28):
            if lib().ob2s_reserve(self.h, nbytes) == 0:
                return nbytes
            nbytes //= 2
        return 0


@dataclass
class Request:
    idx: int
    kind: int
    n: int
    seed: int
    arrival: float
    steps: int = 10
    start: Optional[float] = None
    finish: Optional[float] = None
    iterations: int = 0
    outer: int = 0
    rel: float = 0.0
    checksum: float = 0.0
    solution: object = None


def make_stream(count: int, rate: float, seed: int, adi_frac: float = 0.3,
                pois_n=(64, 2048), adi_n=(32, 192), steps: int = 10,
                heat_frac: float = 0.0, heat_steps: int = 5) -> List[Request]:
    """Seeded request stream: exponential inter-arrival times (rate per
    second; rate <= 0: everything arrives at t = 0), kind by adi_frac (ADI)
    and heat_frac (2D implicit heat, sizes as Poisson), the rest Poisson,
    sizes log-uniform over the ranges.  With heat_frac = 0 the stream is
    the same draw for draw as without the heat kind."""
    rng = random.Random(seed)
    t = 0.0
    out = []
    for k in range(count):
        if rate > 0:
            t += rng.expovariate(rate)
        u = rng.random()
        kind = ADI3D if u < adi_frac else (HEAT2D if u < adi_frac + heat_frac else POISSON2D)
        lo, hi = adi_n if kind == ADI3D else pois_n
        n = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        out.append(Request(k, kind, n, 1000 + k, t,
                           heat_steps if kind == HEAT2D else steps))
    return out


def request_bytes_moved(r: Request, mode: int) -> float:
    """Algorithmic bytes of a finished request.  Poisson / heat, per CG
    iteration: p' = r + beta p and w = A p' read r and p and write p' and w;
    the update pass reads p' and w and updates x (FP64) and r (FP64: 80 B
    per point; mixed, with FP32 r, w, p and the FP64 x: 48 B); per residual
    replacement the FP64 residual pass reads x and b and writes r (24 B).
    ADI: 72 B per point per step (preproc reads u and writes du, the x and y
    solves read and write du, the z solve reads du and updates u)."""
    if r.kind in (POISSON2D, HEAT2D):
        per, outer = (48.0, 24.0) if mode == MIXED else (80.0, 24.0)
        return r.n * r.n * (per * r.iterations + outer * (r.outer + 1))
    return r.n ** 3 * 72.0 * r.steps


def serve(engine: Engine, stream: List[Request], budget_bytes: int, iters: int = 16,
          max_active: int = MAX_ACTIVE, keep_solutions: bool = False) -> Dict:
    """Runs the stream through the engine in real time (arrival times are
    offsets from the start); returns the statistics.  Before the clock
    starts, the engine's memory pool is grown to the HBM budget once (a
    server's start-up), so that admitted requests do not map memory."""
    if hasattr(engine, "reserve_up_to"):
        engine.reserve_up_to(budget_bytes)
    pending = sorted(stream, key=lambda r: r.arrival)
    queue: List[Request] = []
    running: Dict[int, Request] = {}
    used = 0
    done: List[Request] = []
    t0 = time.perf_counter()
    i = 0
    launches0 = engine.launches()
    while i < len(pending) or queue or running:
        now = time.perf_counter() - t0
        while i < len(pending) and pending[i].arrival <= now:
            queue.append(pending[i])
            i += 1
        # admission: arrival order, slots and HBM budget
        while queue and len(running) < max_active:
            r = queue[0]
            need = engine.request_bytes(r.kind, r.n)
            if used + need > budget_bytes and running:
                break
            queue.pop(0)
            rid = engine.submit(r.kind, r.n, r.seed, r.steps)
            r.start = time.perf_counter() - t0
            running[rid] = r
            used += need
        if not running:
            if i < len(pending):  # idle until the next arrival
                time.sleep(max(0.0, pending[i].arrival - (time.perf_counter() - t0)))
            continue
        for rid in engine.run(iters):
            r = running.pop(rid)
            r.finish = time.perf_counter() - t0
            res = engine.result(rid)
            r.iterations, r.outer, r.rel, r.checksum = (res.iterations, res.outer,
                                                         res.rel_residual, res.checksum)
            if keep_solutions:
                r.solution = engine.fetch(rid, r.n ** (3 if r.kind == ADI3D else 2))
            used -= engine.request_bytes(r.kind, r.n)
            engine.release(rid)
            done.append(r)
    wall = time.perf_counter() - t0
    lat = sorted(r.finish - r.arrival for r in done)

    def pct(p):
        return lat[min(len(lat) - 1, int(math.ceil(p / 100.0 * len(lat))) - 1)] if lat else 0.0

    moved = sum(request_bytes_moved(r, engine.mode) for r in done)
    pois = [r for r in done if r.kind in (POISSON2D, HEAT2D)]
    return {
        "requests": len(done), "wall_s": wall, "solves_per_s": len(done) / wall,
        "p50_s": pct(50), "p99_s": pct(99), "mean_s": sum(lat) / max(1, len(lat)),
        "GBps_model": moved / wall / 1e9,
        "max_rel_residual": max([r.rel for r in pois] or [0.0]),
        "launches": engine.launches() - launches0,
        "done": done,
    }


def summary(stats: Dict) -> Dict:
    return {k: v for k, v in stats.items() if k != "done"}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--requests", type=int, default=2000)
    ap.add_argument("--rate", type=float, default=0.0,
                    help="arrivals per second (0: all requests at t = 0)")
    ap.add_argument("--mode", default="both", choices=["mixed", "fp64", "both"])
    ap.add_argument("--budget-gb", type=float, default=160.0)
    ap.add_argument("--iters", type=int, default=16, help="engine iterations per graph replay")
    ap.add_argument("--tile-y", type=int, default=32)
    ap.add_argument("--inner-tol", type=float, default=1e-2,
                    help="residual drop between FP64 residual replacements")
    ap.add_argument("--seed", type=int, default=6)
    ap.add_argument("--min-n", type=int, default=64, help="smallest Poisson grid")
    ap.add_argument("--max-n", type=int, default=2048, help="largest Poisson grid")
    ap.add_argument("--adi-frac", type=float, default=0.3, help="share of ADI requests")
    ap.add_argument("--heat-frac", type=float, default=0.0,
                    help="share of 2D implicit heat requests (5 backward-Euler steps each)")
    a = ap.parse_args(argv)
    stream_args = dict(count=a.requests, rate=a.rate, seed=a.seed, pois_n=(a.min_n, a.max_n),
                       adi_frac=a.adi_frac, heat_frac=a.heat_frac)
    budget = int(a.budget_gb * 1e9)
    out = {"config": {"requests": a.requests, "rate": a.rate, "budget_gb": a.budget_gb,
                      "iters_per_replay": a.iters, "tile_y": a.tile_y,
                      "inner_tol": a.inner_tol, "seed": a.seed, "tol": 1e-8,
                      "poisson_n": [a.min_n, a.max_n], "adi_frac": a.adi_frac,
                      "heat_frac": a.heat_frac,
                      "adi_n": [32, 192], "adi_steps": 10}}
    sols = {}
    if a.mode in ("mixed", "both"):
        e = Engine(MIXED, inner_tol=a.inner_tol, tile_y=a.tile_y)
        st = serve(e, make_stream(**stream_args), budget, a.iters,
                   keep_solutions=a.mode == "both" and a.requests <= 64)
        e.close()
        out["mixed_batched"] = summary(st)
        sols["mixed"] = {r.idx: r for r in st["done"]}
    if a.mode in ("fp64", "both"):
        e = Engine(FP64, inner_tol=a.inner_tol, tile_y=a.tile_y)
        st = serve(e, make_stream(**stream_args), budget, a.iters, max_active=1,
                   keep_solutions=a.mode == "both" and a.requests <= 64)
        e.close()
        out["fp64_one_at_a_time"] = summary(st)
        sols["fp64"] = {r.idx: r for r in st["done"]}
    if a.mode == "both":
        out["speedup_solves_per_s"] = (out["mixed_batched"]["solves_per_s"] /
                                       out["fp64_one_at_a_time"]["solves_per_s"])
        # checksum agreement of every request (solutions when kept)
        worst = 0.0
        for k, rm in sols["mixed"].items():
            rf = sols["fp64"][k]
            if rm.solution is not None and rf.solution is not None:
                import numpy as np
                d = float(np.max(np.abs(rm.solution - rf.solution)) /
                          max(1e-300, float(np.max(np.abs(rf.solution)))))
            else:
                d = abs(rm.checksum - rf.checksum) / max(1e-300, abs(rf.checksum))
            worst = max(worst, d)
        out["mixed_vs_fp64_max_rel_diff"] = worst
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
