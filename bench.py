"""Benchmark: OPS 2D compressible hydro (CloverLeaf application) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--cells 3840] [--no-baseline] [--configs all|none|a,b]

Workload: the CloverLeaf 2D Lagrangian-Eulerian hydro application, unchanged
OPS user code, on 3840 x 3840 cells (ideal gas gamma=1.4, background rho=0.2
e=1.0, a seeded cell-aligned square of 1/16 of the domain at rho=1.0 e=2.5),
FP64.  One step is one hydro time step of the application (~160 par_loops:
timestep/calc_dt min reduction, ideal_gas, viscosity, PdV predictor and
corrector, accelerate, flux_calc, advec_cell / advec_mom sweeps, reset_field
and the 2-deep boundary halo loops).

ours       the app built by the translator on libops_b200.so; steps timed
           with CUDA events on the runtime's work stream; one process per GPU
           under torchrun, each running its own replica (the path does not
           shard across GPUs: replicas only, weak scaling).
reference  the same app on the reference's own OpenMP backend (built from the
           reference sources), all host cores, rank 0 only.

Prints one JSON line (rank 0).  value = cell updates per second over all
ranks (GLUPS).  At N=1 the line also carries `configs`: the multi-block
Poisson, 3D ADI, CG heat and solve-serving configurations, each run in its own
process with its own clock record, HBM fraction and CPU baseline
(apps/config_bench.py).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GLUPS"
UNIT = "GLUPS"
WORKLOAD = "cloverleaf2d_hydro"
FALLBACK_HBM_GBS = 6650.0


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def measured_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            v = float(json.load(f)["hbm_gbs"])
        return v, "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic():
    """Per-launch DRAM bytes of kernels from a committed ncu summary
    (profiles/ncu_traffic.txt: `kernel bytes_per_launch ...`)."""
    out = {}
    p = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    try:
        for line in open(p):
            parts = line.split()
            if len(parts) >= 2 and not line.startswith("#"):
                try:
                    out[parts[0]] = float(parts[1])
                except ValueError:
                    pass
    except OSError:
        pass
    return out


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-i", str(self.idx), "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        self.proc = None
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# multi-process plumbing (torchrun): gloo on CPU tensors only; the GPU work is
# entirely this backend's own, one replica per rank.
# ---------------------------------------------------------------------------
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


def clover_lib(flavour: str) -> str:
    from apps.catalog import artifact, available, build
    # an alternative build of the same app (other code-generation knobs)
    alt = os.environ.get("OPS_B200_CLOVER_LIB")
    if alt and flavour == "b200":
        return alt
    lib = artifact("clover_step", flavour, shared=True)
    if not os.path.exists(lib):
        if not available("clover_step"):
            raise FileNotFoundError("CloverLeaf %s build missing and its sources are not "
                                    "present to build it" % flavour)
        lib = build("clover_step", flavour, shared=True)
    return lib


def cpu_reference_run(cells, steps, warmup, threads, timeout=900):
    """Reference OpenMP backend on the host cores, in its own process."""
    cmd = [sys.executable, "-m", "apps.clover_run", "--flavour", "ref_omp", "--cells",
           str(cells), "--steps", str(steps), "--warmup", str(warmup), "--threads",
           str(threads)]
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="spread",
               OMP_PLACES="cores")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=timeout, env=env)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-2000:])
    line = [l for l in r.stdout.splitlines() if l.startswith("{")][-1]
    return json.loads(line)


def dominant_kernel(report: str):
    rows = []
    for line in report.splitlines():
        p = line.rsplit(" ", 3)
        if len(p) == 4:
            rows.append((p[0], int(p[1]), float(p[2]), float(p[3])))
    if not rows:
        return None, rows
    tot = sum(r[2] for r in rows)
    top = max(rows, key=lambda r: r[2])
    return (top, tot), rows


def run_ours(a, d: Dist):
    """Our arm on this rank's GPU: setup, W warm-up steps, K timed steps."""
    import ctypes
    os.environ["OPS_B200_DEVICE"] = str(d.local)
    lib = clover_lib("b200")
    from apps.clover_run import make_deck
    work = tempfile.mkdtemp(prefix="clover_bench_")
    with open(os.path.join(work, "clover.in"), "w") as f:
        f.write(make_deck(a.cells, a.seed))
    here = os.getcwd()
    os.chdir(work)
    L = ctypes.CDLL(lib, mode=ctypes.RTLD_GLOBAL)
    B = ctypes.CDLL(os.path.join(ROOT, "ops_b200", "lib", "libops_b200.so"),
                    mode=ctypes.RTLD_GLOBAL)
    L.clover_step_run.restype = ctypes.c_double
    B.ob2_launch_count.restype = ctypes.c_longlong
    B.ob2_ktime_report.restype = ctypes.c_size_t
    argv = (ctypes.c_char_p * 2)(b"clover_step", None)
    L.clover_step_setup(1, argv)
    L.clover_step_run(a.warmup)
    B.ob2_dev_sync()
    ev0, ev1 = ctypes.c_void_p(), ctypes.c_void_p()
    B.ob2_event_create(ctypes.byref(ev0))
    B.ob2_event_create(ctypes.byref(ev1))
    n0 = B.ob2_launch_count()
    clocks = ClockSampler(d.local)
    d.barrier()
    clocks.start()
    B.ob2_event_record(ev0)
    h0 = time.perf_counter()
    L.clover_step_run(a.steps)
    host_s = time.perf_counter() - h0  # host time to issue the K steps
    B.ob2_event_record(ev1)
    ms = ctypes.c_float()
    rc = B.ob2_event_elapsed_ms(ev0, ev1, ctypes.byref(ms))
    clk = clocks.stop()
    if rc != 0:
        raise RuntimeError("CUDA error %d in the timed region" % rc)
    launches = B.ob2_launch_count() - n0
    t_ms = d.max(ms.value)
    # per-kernel device times: the same K steps again with an event pair
    # around every launch, kept out of the timed region above (recording
    # ~300 events per step adds host work to every step)
    report = ""
    if a.report:  # lazy-queue statistics (chains, graph replays and updates)
        B.ops_timing_output_str.restype = ctypes.c_size_t
        n = B.ops_timing_output_str(None, 0)
        buf = ctypes.create_string_buffer(n + 1)
        B.ops_timing_output_str(buf, n + 1)
        sys.stderr.write("timed steps: host issue %.3f ms/step, device %.3f ms/step\n%s\n" %
                         (host_s * 1e3 / a.steps, ms.value / a.steps, buf.value.decode()))
    if a.ktime:
        B.ob2_ktime_reset()
        B.ob2_ktime_enable(1)
        L.clover_step_run(a.steps)
        n = B.ob2_ktime_report(None, 0)
        buf = ctypes.create_string_buffer(n + 1)
        B.ob2_ktime_report(buf, n + 1)
        report = buf.value.decode()
        B.ob2_ktime_enable(0)

    # end to end through the C ABI: every dat of the application (the whole
    # hydro state, work arrays and mesh included; interiors, 35 dats) comes in
    # from pinned host buffers with ops_dat_set_data, K steps run, and every
    # dat goes back with ops_dat_fetch_data; host wall clock around all of it.
    L.clover_step_state.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    ndat = L.clover_step_state(0, None, None)
    sizes = (ctypes.c_longlong * ndat)()
    L.clover_step_state(0, None, sizes)
    bufs = (ctypes.c_void_p * ndat)()
    nbytes = 0
    for i in range(ndat):
        p = ctypes.c_void_p()
        B.ob2_host_alloc_pinned(ctypes.byref(p), ctypes.c_size_t(sizes[i]))
        bufs[i] = p.value
        nbytes += sizes[i]
    L.clover_step_state(0, bufs, None)  # current state into the host buffers
    B.ob2_dev_sync()
    d.barrier()
    t0 = time.perf_counter()
    L.clover_step_state(1, bufs, None)
    L.clover_step_run(a.steps)
    L.clover_step_state(0, bufs, None)
    e2e_s = d.max(time.perf_counter() - t0)
    for i in range(ndat):
        B.ob2_host_free_pinned(ctypes.c_void_p(bufs[i]))
    L.clover_step_summary()
    L.clover_step_finish()
    os.chdir(here)
    return {"t_ms": t_ms, "launches": launches, "report": report, "clocks": clk,
            "e2e_s": e2e_s, "e2e_state_bytes": nbytes, "e2e_dats": ndat}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cells", type=int, default=3840)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--no-baseline", action="store_true")
    ap.add_argument("--no-ktime", dest="ktime", action="store_false")
    ap.add_argument("--baseline-steps", type=int, default=2)
    ap.add_argument("--report", action="store_true",
                    help="print the per-kernel device-time table to stderr")
    ap.add_argument("--configs", default="all",
                    help="the other configurations to add under 'configs' (N=1 only): "
                         "all, none, or a comma list of poisson_2x2, adi_256, cg_heat_4096, "
                         "serving")
    a = ap.parse_args(argv)
    if a.warmup < 3:
        a.warmup = 3
    cells_total = float(a.cells) * a.cells
    config = {"workload": WORKLOAD, "cells": "%dx%d" % (a.cells, a.cells), "precision": "fp64",
              "halo_depth": 2, "seed": a.seed,
              "l2": "inputs larger than L2 (about 3 GB of FP64 fields per replica)"}

    if a.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return 0
        cores = host_cores()
        try:
            r = cpu_reference_run(a.cells, a.steps, a.warmup, cores)
        except Exception as e:  # noqa: BLE001
            print(json.dumps({"impl": "reference", "unavailable": str(e).splitlines()[-1][:200]}))
            return 0
        v = cells_total / r["s_per_step"] / 1e9
        line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": r["s_per_step"] * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic (seeded input deck)", "impl": "reference",
                "config": config, "parallelism": "openmp %d threads" % cores,
                "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "reference",
                                 "sample": "%d steps after %d warm-up steps of the full config"
                                           % (a.steps, a.warmup)},
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    d = Dist()
    # the application prints progress on stdout: send the process's stdout to
    # stderr while it runs so that stdout carries only the result line
    sys.stdout.flush()
    saved_stdout = os.dup(1)
    os.dup2(2, 1)
    try:
        res = run_ours(a, d)
    finally:
        sys.stdout.flush()
        os.dup2(saved_stdout, 1)
        os.close(saved_stdout)
    value = cells_total * a.steps * d.world / (res["t_ms"] * 1e-3) / 1e9
    launches = int(d.sum(res["launches"]))
    e2e_v = cells_total * a.steps * d.world / res["e2e_s"] / 1e9
    if d.rank == 0:
        peak, peak_kind = measured_hbm()
        dk, rows = dominant_kernel(res["report"])
        roof = None
        if a.report:
            sys.stderr.write("kernel launches device_ms algorithmic_bytes\n" + res["report"])
        if dk and dk[0][2] > 0:
            (name, cnt, dms, byts), tot = dk
            avg_s = dms * 1e-3 / cnt
            achieved = (byts / cnt) / avg_s / 1e9
            traffic = ncu_traffic().get(name)
            roof = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak,
                    "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": traffic,
                    "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum per "
                                       "launch at this size, from the committed capture "
                                       "profiles/ncu_traffic.txt (not measured in this run)"),
                    "algorithmic_bytes_per_launch": byts / cnt,
                    "avg_launch_us": avg_s * 1e6, "share_of_device_time": dms / tot if tot else None}
            step_bytes = sum(r[3] for r in rows) / a.steps
            roof["step_algorithmic_GBps"] = step_bytes / (res["t_ms"] * 1e-3 / a.steps) / 1e9
            roof["step_frac"] = roof["step_algorithmic_GBps"] / peak
        base = None
        if not a.no_baseline and d.world == 1:
            cores = host_cores()
            try:
                r = cpu_reference_run(a.cells, a.baseline_steps, 1, cores)
                base = {"value": cells_total / r["s_per_step"] / 1e9, "unit": UNIT,
                        "cores": cores, "kind": "reference",
                        "sample": "%d steps (after 1 warm-up) of the %dx%d config on the "
                                  "reference OpenMP backend" % (a.baseline_steps, a.cells, a.cells)}
            except Exception as e:  # noqa: BLE001
                base = {"value": None, "unit": UNIT, "cores": cores, "kind": "reference",
                        "sample": "unavailable: " + str(e).splitlines()[-1][:160]}
        configs = None
        if d.world == 1 and a.configs != "none":
            from apps import config_bench
            names = (list(config_bench.CONFIGS) if a.configs == "all"
                     else [c for c in a.configs.split(",") if c])
            configs = config_bench.run_all(names, ClockSampler(d.local), peak, host_cores(),
                                           baseline=not a.no_baseline)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": d.world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": res["t_ms"] / a.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic (seeded input deck)",
                "config": config, "parallelism": "replicas x%d" % d.world,
                "roofline": roof, "cpu_baseline": base,
                "e2e": {"value": e2e_v, "unit": UNIT,
                        "h2d_bytes_per_step": res["e2e_state_bytes"] / a.steps,
                        "d2h_bytes_per_step": res["e2e_state_bytes"] / a.steps,
                        "note": "all %d dats of the application (%.2f GB) set from pinned host "
                                "buffers before and fetched back after the K steps "
                                "(ops_dat_set_data / ops_dat_fetch_data)"
                                % (res["e2e_dats"], res["e2e_state_bytes"] / 1e9)},
                "gpu_launches": launches, "clocks": res["clocks"]}
        if configs is not None:
            line["configs"] = configs
        print(json.dumps(line), flush=True)
    d.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
