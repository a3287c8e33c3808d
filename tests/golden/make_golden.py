"""Generate tests/golden/golden.json: outputs of the REFERENCE OPS backend
itself, used to pin the CPU oracle and the GPU path.

Run in a checkout where the reference tree is available (it is read at build
time only):

    python tests/golden/make_golden.py

Contents
  * known answers that the reference's own tests assert, with the file:line
    they come from (Poisson defaults, CloverLeaf test problems 1 and 2,
    Laplace step7);
  * the printed results of this repository's drivers (multi-block Poisson,
    opsunit, CG heat conduction) when built on the reference's sequential
    backend (ref_seq).
"""

from __future__ import annotations

import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def run(exe, args=(), cwd=None):
    r = subprocess.run([exe, *args], capture_output=True, text=True, cwd=cwd, timeout=1800)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-2000:])
    return r.stdout


def numbers(text, key):
    out = []
    for line in text.splitlines():
        if line.startswith(key):
            out.append([float(x) if any(c in x for c in ".e") else int(x)
                        for x in line.split()[1:] if x.lstrip("-").replace(".", "").replace(
                            "e", "").replace("+", "").replace("-", "").isdigit()])
    return out


def main():
    from apps import catalog
    g = {
        "known_answers": {
            "ref_poisson_default_total_error": {
                "value": 16.5173570176708,
                "source": "apps/c/poisson/poisson.cpp:307-316 (20x20, 10 iterations)"},
            "cloverleaf_test1_ke": {
                "value": 1.82280367310258,
                "source": "apps/c/CloverLeaf/field_summary.cpp:91 (clover.in_default)"},
            "cloverleaf_test2_ke": {
                "value": 1.19316898756307,
                "source": "apps/c/CloverLeaf/field_summary.cpp:92 (clover_bm_short.in)"},
            "laplace_step7_error": {
                "value": 2.421354960840227e-03,
                "source": "apps/c/laplace2d_tutorial/step7/laplace2d.cpp:134 (4094^2, 100 it)"},
        },
        "reference_runs": {},
    }
    cases = {
        "poisson_mb_default": ("poisson_mb", []),
        "poisson_mb_3x3": ("poisson_mb", ["-nb=3", "-n=40", "-sweeps=300", "-check=50"]),
        "opsunit_default": ("opsunit", []),
        "opsunit_29x17": ("opsunit", ["-nx=29", "-ny=17"]),
        "heat_cg_128": ("heat_cg", ["-n=128"]),
        "heat_cg_96_fixed": ("heat_cg", ["-n=96", "-dt=2e-4", "-tol=0", "-maxit=40"]),
    }
    for key, (name, args) in cases.items():
        exe = catalog.build(name, "ref_seq")
        out = run(exe, args)
        lines = [l for l in out.splitlines()
                 if l.split() and l.split()[0] in ("sweep", "checksum", "sums", "min", "max",
                                                   "count", "fetch_b", "fp64", "mixed",
                                                   "compare")]
        g["reference_runs"][key] = {"app": name, "args": args, "backend": "reference ref_seq",
                                    "lines": lines}
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(g, f, indent=1)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    main()
