"""The oracle's halo transfer and tridiagonal solve, driven through the same C
ABI as the GPU tests, against the numpy restatements those tests use (CPU).
Run in a child process: the oracle library exports the same symbols as
libops_b200.so."""

import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import sys, ctypes as C, numpy as np
sys.path.insert(0, %r)
import tests.cabi as cabi
cabi.LIB = %r
from tests.test_gpu_cabi import CASES_2D, np_halo, np_trid
L = cabi.lib()
for case in range(len(CASES_2D)):
    for types in [("double", "double"), ("float", "float"), ("double", "float")]:
        b0 = L.ops_decl_block(2, b"a"); b1 = L.ops_decl_block(2, b"b")
        src = cabi.Dat(b0, 2, [12, 20], [-2, -2], [2, 2], types[0], "s")
        dst = cabi.Dat(b1, 2, [20, 14], [-2, -2], [2, 2], types[1], "d")
        rng = np.random.default_rng(case)
        s = rng.standard_normal(src.full_shape()).astype(src.dtype)
        d = rng.standard_normal(dst.full_shape()).astype(dst.dtype)
        src.set_full(s); dst.set_full(d)
        it, fb, tb, fd, td = CASES_2D[case]
        h = L.ops_decl_halo(src.h, dst.h, cabi.ivec(it), cabi.ivec(fb), cabi.ivec(tb),
                            cabi.ivec(fd), cabi.ivec(td))
        L.ops_halo_transfer(L.ops_decl_halo_group(1, (C.c_void_p * 1)(h)))
        assert np.array_equal(dst.get_full(), np_halo(s, d, src.d_m, dst.d_m, it, fb, tb, fd, td)), case
blk = L.ops_decl_block(3, b"t")
for solvedim in range(3):
    for inc in (False, True):
        nx, ny, nz = 9, 7, 5
        ds = {k: cabi.Dat(blk, 3, [nx, ny, nz], [-1, -1, -1], [1, 1, 1], "double", k) for k in "abcdu"}
        rng = np.random.default_rng(solvedim)
        full = ds["a"].full_shape()
        v = {"a": rng.uniform(-1, 1, full), "c": rng.uniform(-1, 1, full),
             "b": 3 + rng.uniform(0, 1, full), "d": rng.uniform(-1, 1, full),
             "u": rng.uniform(-1, 1, full)}
        for k in "abcdu": ds[k].set_full(v[k])
        box = [1, nx - 1, 2, ny, 0, nz]
        if inc:
            L.ops_tridMultiDimBatch_Inc(3, solvedim, cabi.ivec(box), ds["a"].h, ds["b"].h,
                                        ds["c"].h, ds["d"].h, ds["u"].h, None)
            got = ds["u"].get_full()
        else:
            L.ops_tridMultiDimBatch(3, solvedim, cabi.ivec(box), ds["a"].h, ds["b"].h,
                                    ds["c"].h, ds["d"].h, None)
            got = ds["d"].get_full()
        want = np_trid(v["a"], v["b"], v["c"], v["d"], v["u"] if inc else None, solvedim,
                       [b + 1 for b in box])
        assert np.max(np.abs(got - want)) < 1e-13, (solvedim, inc)
print("ok")
"""


def test_oracle_halo_and_trid_match_numpy_models():
    sys.path.insert(0, ROOT)
    from apps.catalog import ensure_oracle_lib
    lib = ensure_oracle_lib()
    r = subprocess.run([sys.executable, "-c", SCRIPT % (ROOT, lib)], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0 and "ok" in r.stdout, r.stderr[-3000:]
