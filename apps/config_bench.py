"""The four other configurations of the benchmark record, each run in its own
process on this backend, with its own clock record, HBM fraction and CPU
baseline:

  poisson_2x2   multi-block Poisson Jacobi, 2 x 2 blocks of 256^2, 1000 sweeps
                with a max-abs residual reduction every 100 (apps/poisson_mb)
  adi_256       3D ADI heat, 256^3, 50 steps, FP64 and FP32 storage with FP64
                elimination (apps/adi3d)
  cg_heat_4096  CG heat conduction, 4096^2, to 1e-10 relative residual, FP64
                CG and the mixed form (apps/heat_cg)
  serving       2000 Poisson / ADI solve requests, mixed-precision batched
                engine against one-at-a-time FP64 (ops_b200.serving), all at
                t = 0, and a Poisson-arrival run at the FP64 engine's capacity

CPU baselines: the reference's own sequential backend (OpenMP-parallel
par_loops, all host cores) for poisson_2x2 (full config) and cg_heat_4096
(a bounded sample of CG iterations, scaled to the FP64 iteration count); the
CPU restatement of the Thomas solves for adi_256 (the reference's
tridiagonal solver is an external library absent from its tree), one step.
The serving configuration's baseline is its own FP64 one-at-a-time run.

  reference_cuda_cloverleaf   the headline CloverLeaf configuration on the
                reference's own CUDA backend on the same GPU (context only)
"""

from __future__ import annotations

import json
import os
import re
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(cmd, env=None, timeout=1800):
    t0 = time.perf_counter()
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=timeout,
                       env=dict(os.environ, PYTHONPATH=ROOT, **(env or {})))
    if r.returncode != 0:
        raise RuntimeError("%s failed (rc %d): %s" % (" ".join(cmd[:4]), r.returncode,
                                                      r.stderr[-600:]))
    return r.stdout, time.perf_counter() - t0


def _num(pattern, text, cast=float):
    m = re.search(pattern, text)
    if not m:
        raise RuntimeError("no match for %r" % pattern)
    return cast(m.group(1))


def _frac(gbps, peak):
    return gbps / peak if peak else None


def poisson_2x2(clock, peak, cores, baseline=True):
    clock.start()
    out, _ = _run([sys.executable, "-m", "apps.run_shared", "poisson_mb", "b200"])
    clk = clock.stop()
    glups = _num(r"sweeps\s+\d+\s+time\s+\S+\s+s\s+(\S+)\s+GLUPS", out)
    # Jacobi loop (u READ 5-point, f READ, u2 WRITE: 24 B per point) + copy
    # back (16 B per point) per sweep, the transfer model's bytes
    gbps = glups * 40.0
    e = {"metric": "GLUPS", "value": glups, "unit": "GLUPS", "clocks": clk,
         "workload": "poisson_mb: 2x2 blocks of 256^2, FP64 5-point Jacobi, 1000 sweeps, "
                     "ops_halo_transfer every sweep, OPS_MAX residual every 100",
         "roofline": {"bound": "l2", "achieved": gbps, "unit": "GB/s", "peak": peak,
                      "frac": _frac(gbps, peak),
                      "note": "6 MB working set stays in the 126 MB L2: launch- and "
                              "latency-bound, the HBM fraction is not the bound"}}
    if baseline:
        exe = os.path.join(ROOT, "oracle", "_ref", "apps", "poisson_mb", "ref_seq", "poisson_mb")
        try:
            cout, _ = _run([exe], env={"OMP_NUM_THREADS": str(cores)})
            e["cpu_baseline"] = {"value": _num(r"sweeps\s+\d+\s+time\s+\S+\s+s\s+(\S+)\s+GLUPS",
                                               cout),
                                 "unit": "GLUPS", "cores": cores, "kind": "reference",
                                 "sample": "full config on the reference's sequential backend "
                                           "(libops_seq, OpenMP par_loops)"}
        except Exception as ex:  # noqa: BLE001
            e["cpu_baseline"] = {"value": None, "sample": "unavailable: %s" % str(ex)[:160]}
    return e


def adi_256(clock, peak, cores, baseline=True):
    clock.start()
    out, _ = _run([sys.executable, "-m", "apps.run_shared", "adi3d", "b200", "-n=256",
                   "-steps=50", "-prec=both"])
    clk = clock.stop()
    ms64 = _num(r"fp64\s+\d+\s+steps\s+\S+\s+s\s+(\S+)\s+ms/step", out)
    ms32 = _num(r"fp32\s+\d+\s+steps\s+\S+\s+s\s+(\S+)\s+ms/step", out)
    err = _num(r"relative L2 error\s+(\S+)", out)
    pts = 256.0 ** 3
    g64, g32 = pts * 216.0 / (ms64 * 1e-3) / 1e9, pts * 108.0 / (ms32 * 1e-3) / 1e9
    e = {"metric": "ms/step", "value": ms64, "unit": "ms/step", "higher_is_better": False,
         "fp32_storage_ms_per_step": ms32, "fp32_vs_fp64_rel_l2_error": err, "clocks": clk,
         "workload": "adi3d: 256^3, lambda 1, 50 steps; per step the 7-point preproc "
                     "par_loop and three ops_tridMultiDimBatch solves (x, y, z with add)",
         "roofline": {"bound": "hbm", "achieved": g64, "unit": "GB/s", "peak": peak,
                      "frac": _frac(g64, peak), "fp32_achieved": g32,
                      "fp32_frac": _frac(g32, peak),
                      "bytes": "216 B per point per step FP64, 108 FP32 storage"}}
    if baseline:
        try:
            cout, _ = _run([sys.executable, "-m", "apps.run_shared", "adi3d", "oracle",
                            "-n=256", "-steps=1", "-prec=64"])
            e["cpu_baseline"] = {"value": _num(r"fp64\s+\d+\s+steps\s+\S+\s+s\s+(\S+)\s+ms/step",
                                               cout),
                                 "unit": "ms/step", "cores": 1, "kind": "port",
                                 "sample": "one FP64 step of the full config on the CPU "
                                           "restatement (sequential Thomas per line)"}
        except Exception as ex:  # noqa: BLE001
            e["cpu_baseline"] = {"value": None, "sample": "unavailable: %s" % str(ex)[:160]}
    return e


def cg_heat_4096(clock, peak, cores, baseline=True):
    clock.start()
    out, _ = _run([sys.executable, "-m", "apps.run_shared", "heat_cg", "b200"])
    clk = clock.stop()
    it64 = _num(r"fp64 iterations\s+(\d+)", out, int)
    itm = _num(r"mixed iterations\s+(\d+)", out, int)
    t64 = _num(r"timing fp64\s+(\S+)\s+s", out)
    tm = _num(r"timing mixed\s+(\S+)\s+s", out)
    g64 = _num(r"timing fp64\s+\S+\s+s\s+(\S+)\s+GB/s", out)
    gm = _num(r"timing mixed\s+\S+\s+s\s+(\S+)\s+GB/s", out)
    e = {"metric": "s to 1e-10", "value": t64, "unit": "s", "higher_is_better": False,
         "fp64_iterations": it64, "fp64_true_rel_residual":
             _num(r"fp64 iterations.*true_resid\s+(\S+)", out),
         "mixed_s": tm, "mixed_iterations": itm,
         "mixed_replacements": _num(r"replacements\s+(\d+)", out, int),
         "mixed_true_rel_residual": _num(r"mixed iterations.*true_resid\s+(\S+)", out),
         "mixed_vs_fp64_max_rel_diff": _num(r"compare max_rel_diff\s+(\S+)", out),
         "speedup_mixed_over_fp64": t64 / tm, "clocks": clk,
         "workload": "heat_cg: 4096^2, TeaLeaf operator, two-region conductivity, "
                     "unpreconditioned CG to 1e-10 relative residual",
         "roofline": {"bound": "hbm", "achieved": g64, "unit": "GB/s", "peak": peak,
                      "frac": _frac(g64, peak), "mixed_achieved": gm,
                      "mixed_frac": _frac(gm, peak),
                      "bytes": "104 B per cell per CG iteration FP64, 60 mixed"}}
    if baseline:
        exe = os.path.join(ROOT, "oracle", "_ref", "apps", "heat_cg", "ref_seq", "heat_cg")
        k = 8
        try:
            cout, _ = _run([exe, "-tol=0", "-maxit=%d" % k, "-prec=64"],
                           env={"OMP_NUM_THREADS": str(cores)})
            s_it = _num(r"timing fp64\s+(\S+)\s+s", cout) / k
            e["cpu_baseline"] = {"value": s_it * it64, "unit": "s", "cores": cores,
                                 "kind": "reference",
                                 "sample": "%d FP64 CG iterations at 4096^2 on the reference's "
                                           "sequential backend, %.3f s per iteration, scaled to "
                                           "the %d iterations of the FP64 solve" % (k, s_it, it64)}
        except Exception as ex:  # noqa: BLE001
            e["cpu_baseline"] = {"value": None, "sample": "unavailable: %s" % str(ex)[:160]}
    return e


def serving(clock, peak, cores, baseline=True, requests=2000, rate_requests=600):
    clock.start()
    out, _ = _run([sys.executable, "-m", "ops_b200.serving", "--requests", str(requests),
                   "--mode", "both"], timeout=3600)
    clk = clock.stop()
    r = json.loads([l for l in out.splitlines() if l.startswith("{")][-1])
    m, f = r["mixed_batched"], r["fp64_one_at_a_time"]
    keep = ("requests", "wall_s", "solves_per_s", "p50_s", "p99_s", "GBps_model",
            "max_rel_residual")
    e = {"metric": "solves/s", "value": m["solves_per_s"], "unit": "solves/s",
         "mixed_batched": {k: m[k] for k in keep},
         "fp64_one_at_a_time": {k: f[k] for k in keep},
         "speedup_solves_per_s": r["speedup_solves_per_s"],
         "mixed_vs_fp64_max_rel_diff": r["mixed_vs_fp64_max_rel_diff"], "clocks": clk,
         "workload": "2000 requests all at t = 0: 70 % 2D Poisson n in [64, 2048], 30 % 3D "
                     "ADI n in [32, 192] (log-uniform, seed 6), 1e-8 relative residual, "
                     "160 GB HBM budget",
         "roofline": {"bound": "hbm", "achieved": m["GBps_model"], "unit": "GB/s", "peak": peak,
                      "frac": _frac(m["GBps_model"], peak),
                      "note": "bytes model of the served requests over the run's wall time"}}
    # a Poisson-arrival stream at the FP64 one-at-a-time capacity
    rate = f["solves_per_s"]
    clock.start()
    out, _ = _run([sys.executable, "-m", "ops_b200.serving", "--requests", str(rate_requests),
                   "--rate", "%.3f" % rate, "--mode", "both"], timeout=3600)
    clk2 = clock.stop()
    r2 = json.loads([l for l in out.splitlines() if l.startswith("{")][-1])
    e["arrivals_at_fp64_capacity"] = {
        "requests": rate_requests, "rate_per_s": rate, "clocks": clk2,
        "mixed_batched": {k: r2["mixed_batched"][k] for k in keep},
        "fp64_one_at_a_time": {k: r2["fp64_one_at_a_time"][k] for k in keep}}
    e["cpu_baseline"] = {"value": None, "unit": "solves/s", "cores": cores, "kind": "port",
                         "sample": "none: the configuration's baseline is the FP64 "
                                   "one-at-a-time engine on the same GPU (fp64_one_at_a_time)"}
    return e


def reference_cuda_cloverleaf(clock, peak, cores, baseline=True, cells=3840, steps=20,
                              warmup=5):
    """Context, not a baseline of the record: the headline CloverLeaf
    configuration on the reference's own CUDA backend (its legacy
    translator's CUDA kernels and libops_cuda, built from the reference
    sources for sm_100 with its default flags), on this GPU, host wall clock
    around the steps with a device synchronisation at both ends."""
    clock.start()
    out, _ = _run([sys.executable, "-m", "apps.clover_run", "--flavour", "ref_cuda", "--cells",
                   str(cells), "--steps", str(steps), "--warmup", str(warmup)])
    clk = clock.stop()
    r = json.loads([l for l in out.splitlines() if l.startswith("{")][-1])
    ms = r["s_per_step"] * 1e3
    return {"metric": "GLUPS", "value": cells * cells / (ms * 1e-3) / 1e9, "unit": "GLUPS",
            "ms_per_step": ms, "clocks": clk, "summary": r["summary"],
            "workload": "cloverleaf2d_hydro %dx%d, %d steps after %d warm-up steps, the "
                        "reference's CUDA backend on this GPU (context for the headline line)"
                        % (cells, cells, steps, warmup)}


CONFIGS = {"poisson_2x2": poisson_2x2, "adi_256": adi_256, "cg_heat_4096": cg_heat_4096,
           "serving": serving, "reference_cuda_cloverleaf": reference_cuda_cloverleaf}


def run_all(names, clock, peak, cores, baseline=True):
    out = {}
    for n in names:
        try:
            out[n] = CONFIGS[n](clock, peak, cores, baseline)
        except Exception as ex:  # noqa: BLE001
            try:
                clock.stop()
            except Exception:  # noqa: BLE001
                pass
            out[n] = {"error": str(ex)[:400]}
    return out
