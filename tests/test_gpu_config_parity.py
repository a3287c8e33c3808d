"""Parity at the full configuration sizes: the b200 build of each
configuration against a CPU build of the same program on the same seeded
inputs, every dat compared element by element.

* CloverLeaf 2D hydro, 3840^2 cells, 5 steps: this backend against the
  reference's own OpenMP backend (its legacy translator and libops_seq, built
  from the reference sources).  Every dat's interior is read through
  ops_dat_fetch_data on both sides (apps/dumpdats.h); the field summary
  (volume, mass, pressure, internal and kinetic energy sums) is compared too.
* 3D ADI heat, 256^3, 3 steps, FP64 and FP32 storage: this backend against
  the CPU oracle (the reference's tridiagonal solve lives in the external
  tridsolver library, which the reference tree does not contain, so the
  oracle's Thomas restatement is the checker for the solves).
* CG heat conduction, 4096^2, 40 CG iterations (tolerance 0, so the count is
  fixed) in the FP64 and the mixed form: this backend against the reference's
  own sequential backend (ref_seq build of the driver), dats through
  ops_dat_fetch_data.

Tolerances: integer dats bit-exact; FP64 dats 1e-12 relative per element
(|a-b| / max(|b|, 1e-3 max|b|)); FP32-stored dats 1e-6 (a float rounding of
an FP64 value computed in another order); reductions 1e-11 relative.
"""

import json
import os
import re
import subprocess
import sys

import pytest

from tests.apprun import ROOT, assert_lines_close, ensure, result_lines, run_app
from tests.opsdump import compare, read_dump

pytestmark = pytest.mark.gpu


def check(gpu_dump, cpu_dump, tol=1e-12, float_tol=1e-6):
    diffs = compare(gpu_dump, cpu_dump, mmap=True)
    meta = read_dump(cpu_dump, mmap=True)
    bad = {n: d for n, d in diffs.items()
           if d > (float_tol if meta[n][0]["type"] == "float" else tol)}
    assert diffs and not bad, bad
    return diffs


def test_cloverleaf_3840_matches_reference_openmp(tmp_path):
    ensure("clover_step", "b200")
    ensure("clover_step", "ref_omp")
    res, dumps = {}, {}
    for fl in ("b200", "ref_omp"):
        dumps[fl] = str(tmp_path / ("%s.dump" % fl))
        r = subprocess.run([sys.executable, "-m", "apps.clover_run", "--flavour", fl, "--cells",
                            "3840", "--steps", "5", "--fetch-dump", dumps[fl]], cwd=ROOT,
                           capture_output=True, text=True, timeout=1200)
        assert r.returncode == 0, r.stderr[-2000:]
        res[fl] = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
    try:
        diffs = check(dumps["b200"], dumps["ref_omp"])
        print("PARITY cloverleaf_3840 per element", json.dumps(diffs, sort_keys=True))
        assert len(diffs) == 35
    finally:
        for p in dumps.values():
            if os.path.exists(p):
                os.unlink(p)
    sg, sr = res["b200"]["summary"], res["ref_omp"]["summary"]
    assert sg["step"] == sr["step"] == 5
    for k in ("volume", "mass", "pressure", "ie", "ke"):
        assert abs(sg[k] - sr[k]) <= 1e-11 * abs(sr[k]), (k, sg[k], sr[k])


@pytest.mark.parametrize("prec", ["64", "32"])
def test_adi_256_matches_oracle(prec, tmp_path):
    """The state u per element (1e-12 FP64, 1e-6 FP32 storage); du, the
    right-hand side the three solves overwrite, relative to its field's scale
    (1e-12 of max|du|): the chunked Thomas/PCR elimination rounds in another
    order than the oracle's sequential Thomas sweep, which shows per element
    on du's near-zero values (5e-12 of the element at 1e-3 of the scale,
    i.e. 5e-15 of the scale) but stays at round-off of the field."""
    args = ["-n=256", "-steps=3", "-prec=" + prec]
    try:
        gout, gd = run_app("adi3d", "b200", args, dump=True)
        cout, cd = run_app("adi3d", "oracle", args, dump=True)
        diffs = compare(gd, cd, mmap=True, skip=("du_",))
        meta = read_dump(cd, mmap=True)
        for name, d in diffs.items():
            assert d <= (1e-6 if meta[name][0]["type"] == "float" else 1e-12), (name, d)
        dd = compare(gd, cd, mmap=True, floor_frac=1.0)
        print("PARITY adi_256 prec %s per element" % prec, json.dumps(diffs, sort_keys=True),
              "relative to scale", json.dumps(dd, sort_keys=True))
        for name, d in dd.items():
            if name.startswith("du_"):
                assert d <= (1e-6 if meta[name][0]["type"] == "float" else 1e-12), (name, d)
    finally:
        for p in (locals().get("gd"), locals().get("cd")):
            if p and os.path.exists(p):
                os.unlink(p)
    key = "fp64" if prec == "64" else "fp32"
    g = [l for l in result_lines(gout, (key,)) if "checksum" in l]
    c = [l for l in result_lines(cout, (key,)) if "checksum" in l]
    assert_lines_close(g, c, 1e-11 if prec == "64" else 1e-6)


@pytest.mark.parametrize("prec", ["64", "32"])
def test_heat_cg_4096_matches_reference_seq(prec, tmp_path):
    """The dot products are summed in another order than the reference's
    sequential backend does (a fixed-order tree against a running sum), so
    alpha and beta move by an ulp and the Krylov vectors r, p, w pick up
    round-off that the 40 iterations amplify: compared relative to each
    field's scale (FP64 1e-10, FP32 vectors 1e-4), the FP64 iterate u per
    element (1e-11) and the mixed form's FP64 iterate x relative to its
    scale (1e-6); the set-up dats (density, u0, conductivities) exactly; the
    iteration and replacement counts exactly, the checksums of the solution
    (reductions) within 1e-11 (FP64) and 1e-6 (mixed)."""
    import numpy as np
    exe = ensure("heat_cg", "ref_seq", shared=False)
    gd, cd = str(tmp_path / "b200.dump"), str(tmp_path / "ref.dump")
    args = ["-n=4096", "-tol=0", "-maxit=40", "-prec=" + prec]
    try:
        gout, _ = run_app("heat_cg", "b200", args + ["-dump=" + gd])
        r = subprocess.run([exe, *args, "-dump=" + cd], capture_output=True, text=True,
                           timeout=1800)
        assert r.returncode == 0, r.stderr[-2000:]
        cout = r.stdout
        per_elem = compare(gd, cd, mmap=True)
        scale = compare(gd, cd, mmap=True, floor_frac=1.0)
    finally:
        for p in (gd, cd):
            if os.path.exists(p):
                os.unlink(p)
    print("PARITY heat_cg_4096 prec %s per element" % prec, json.dumps(per_elem, sort_keys=True),
          "relative to scale", json.dumps(scale, sort_keys=True))
    for name in ("density", "u0", "Kx", "Ky", "Kx32", "Ky32"):
        if name in per_elem:
            assert per_elem[name] == 0.0, (name, per_elem[name])
    if prec == "64":
        assert per_elem["u"] <= 1e-11, per_elem
        for name in ("r", "p", "w"):
            assert scale[name] <= 1e-10, (name, scale[name])
    else:
        assert scale["x"] <= 1e-6, scale
        for name in ("r32", "p32", "w32"):
            assert scale[name] <= 1e-4, (name, scale[name])
    key = "fp64" if prec == "64" else "mixed"
    g = [l for l in result_lines(gout, (key,)) if "iterations" in l or "checksum" in l]
    c = [l for l in result_lines(cout, (key,)) if "iterations" in l or "checksum" in l]
    assert len(g) == 2, gout[-1000:]
    words = lambda l: [t for t in l.split() if not re.search(r"[.eE]\d|\d[.eE]", t)]
    assert [words(l) for l in g] == [words(l) for l in c]
    ck = lambda lines: [float(l.split()[-1]) for l in lines if "checksum" in l][0]
    assert abs(ck(g) - ck(c)) <= (1e-11 if prec == "64" else 1e-6) * abs(ck(c))
