"""GPU parity of whole OPS programs: the b200 build against the CPU oracle on
the same inputs, dat by dat (halos included), and the reference's known
answers on the b200 build.

Tolerances: integer dats bit-exact; FP64 dats 1e-12 relative per element
(the generated kernels use IEEE arithmetic without FMA contraction, so in
practice they are bit-identical); reductions 1e-11 relative; FP32-storage dats
1e-6 relative (one float rounding of an FP64 value that was computed in a
different order).
"""

import os
import re
import tempfile

import pytest

from tests.apprun import (assert_lines_close, clover_deck_test1, clover_deck_test2,
                          result_lines, run_app, run_exe)
from tests.opsdump import compare

pytestmark = pytest.mark.gpu


def check_dumps(gpu_dump, cpu_dump, tol=1e-12, float_tol=1e-6, skip=(), floor_frac=1e-3):
    from tests.opsdump import read_dump
    diffs = compare(gpu_dump, cpu_dump, skip=skip, floor_frac=floor_frac)
    meta = read_dump(cpu_dump)
    bad = {}
    for name, d in diffs.items():
        t = float_tol if meta[name][0]["type"] == "float" else tol
        if d > t:
            bad[name] = d
    assert not bad, bad
    return diffs


@pytest.mark.parametrize("args", [[], ["-nx=29", "-ny=17"], ["-nx=130", "-ny=7"],
                                  ["-nx=31", "-ny=19", "-soa=1"]])
def test_opsunit_parity(args, golden):
    gout, gd = run_app("opsunit", "b200", args, dump=True)
    cout, cd = run_app("opsunit", "oracle", args, dump=True)
    check_dumps(gd, cd)
    assert_lines_close(result_lines(gout), result_lines(cout), 1e-11)
    if not args:
        want = golden["reference_runs"]["opsunit_default"]["lines"]
        got = [l for l in result_lines(gout) if l.split()[0] in ("sums", "min", "max", "count",
                                                                  "fetch_b")]
        assert_lines_close(got, want, 1e-11)


@pytest.mark.parametrize("args", [[], ["-n=9"]])
def test_hdunit_5d_parity(args):
    """A 5D block (apps/hdunit): a fill from the point index over the whole
    storage, a stencil reaching one point along each of the five axes, sum
    and max reductions over the 5D range (the 3rd to 5th axes folded into
    the grid's z index), and a halo group flipped along the 4th and 5th
    axes: every dat bit-exact against the oracle, and the printed sums and
    maxima equal (their values are sums of dyadic numbers, exact in any
    order; the oracle's were checked against a numpy restatement)."""
    gout, gd = run_app("hdunit", "b200", args, dump=True)
    cout, cd = run_app("hdunit", "oracle", args, dump=True)
    diffs = compare(gd, cd)
    assert diffs and max(diffs.values()) == 0.0, diffs
    g = [l for l in gout.splitlines() if l.startswith("hdunit")]
    c = [l for l in cout.splitlines() if l.startswith("hdunit")]
    assert len(g) == 2 and g == c, (g, c)
    if not args:
        assert g[0] == "hdunit sums 63731.25 max 107.34375", g


def test_poisson_mb_parity_and_reference(golden):
    gout, gd = run_app("poisson_mb", "b200", dump=True)
    cout, cd = run_app("poisson_mb", "oracle", dump=True)
    check_dumps(gd, cd)
    want = golden["reference_runs"]["poisson_mb_default"]["lines"]
    assert_lines_close(result_lines(gout), want, 1e-11)


def test_poisson_mb_3x3_ragged(golden):
    g = golden["reference_runs"]["poisson_mb_3x3"]
    gout, gd = run_app("poisson_mb", "b200", g["args"], dump=True)
    cout, cd = run_app("poisson_mb", "oracle", g["args"], dump=True)
    check_dumps(gd, cd)
    assert_lines_close(result_lines(gout), g["lines"], 1e-11)


@pytest.mark.parametrize("args", [["-n=24", "-steps=5", "-prec=both"],
                                  ["-nx=33", "-ny=17", "-nz=20", "-steps=3", "-prec=both"],
                                  ["-nx=300", "-ny=9", "-nz=6", "-steps=2", "-prec=64"]])
def test_adi3d_parity(args):
    """The solves use a different elimination order than the oracle's Thomas
    sweep (chunked Thomas + PCR), so agreement is at round-off relative to the
    field's scale: |gpu - oracle| <= 1e-12 * max|oracle| per dat (FP64), and
    one float rounding for FP32 storage."""
    gout, gd = run_app("adi3d", "b200", args, dump=True)
    cout, cd = run_app("adi3d", "oracle", args, dump=True)
    check_dumps(gd, cd, tol=1e-12, float_tol=1e-6, floor_frac=1.0)
    assert_lines_close(result_lines(gout, ("fp64",))[:1], result_lines(cout, ("fp64",))[:1], 1e-11)


def test_cloverleaf_fields_match_oracle(tmp_path):
    import json
    import subprocess
    import sys
    from tests.apprun import ensure, ROOT
    ensure("clover_step", "b200")
    ensure("clover_step", "oracle")
    dumps = {}
    for fl in ("b200", "oracle"):
        dumps[fl] = str(tmp_path / ("%s.dump" % fl))
        r = subprocess.run([sys.executable, "-m", "apps.clover_run", "--flavour", fl, "--cells",
                            "96", "--steps", "15", "--dump", dumps[fl]], cwd=ROOT,
                           capture_output=True, text=True, timeout=900)
        assert r.returncode == 0, r.stderr[-2000:]
    check_dumps(dumps["b200"], dumps["oracle"])


def test_reference_poisson_on_b200(golden):
    out = run_exe("ref_poisson", "b200")
    v = float(re.search(r"Total error: (\S+)", out).group(1))
    want = golden["known_answers"]["ref_poisson_default_total_error"]["value"]
    assert abs(v - want) <= 1e-12 * want and "PASSED" in out


def test_reference_laplace_on_b200(golden):
    out = run_exe("ref_laplace", "b200")
    assert "PASSED" in out, out[-500:]


@pytest.mark.parametrize("deck", ["test1", "test2"])
def test_reference_cloverleaf_known_answers_on_b200(deck):
    d = tempfile.mkdtemp(prefix="clover_%s_" % deck)
    with open(os.path.join(d, "clover.in"), "w") as f:
        f.write(clover_deck_test1() if deck == "test1" else clover_deck_test2())
    out = run_exe("cloverleaf", "b200", cwd=d)
    assert "This test is considered PASSED" in out, out[-800:]


def test_reference_mblock_halos_match_oracle(tmp_path):
    """mblock (reference app): multi-block halo transfers with flipped and
    permuted orientations; every dat compared with the oracle."""
    import subprocess
    from tests.apprun import ensure
    dumps = {}
    for fl in ("b200", "oracle"):
        exe = ensure("ref_mblock", fl, shared=False)
        dumps[fl] = str(tmp_path / ("%s.dump" % fl))
        r = subprocess.run([exe], cwd=str(tmp_path), capture_output=True, text=True,
                           env=dict(os.environ, OPS_DUMP_FILE=dumps[fl]), timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
    diffs = compare(dumps["b200"], dumps["oracle"])
    assert max(diffs.values()) == 0.0, diffs


HEAT_KEYS = ("fp64", "mixed", "compare")


def words_and_counts(line):
    """the line's words and integer fields (iteration counts), without the
    floating-point values"""
    return [t for t in line.split() if not re.search(r"[.eE]\d|\d[.eE]", t)]


def test_heat_cg_fixed_iterations_match_oracle(golden):
    """40 CG iterations without a stopping test, FP64 and mixed: the dats
    against the oracle's.  The dot products are summed in a different order
    (tree vs sequential), so alpha and beta differ in the last bits and the
    iterates drift apart at round-off: the FP64 solver's dats (and the set-up
    dats) within 1e-10 of the field's scale; the mixed form's dats (FP32
    vectors and the FP64 iterate they update) within 1e-5 of the field's
    scale (a beta that rounds to the other float moves every point by one
    float ulp)."""
    g = golden["reference_runs"]["heat_cg_96_fixed"]
    gout, gd = run_app("heat_cg", "b200", g["args"], dump=True)
    cout, cd = run_app("heat_cg", "oracle", g["args"], dump=True)
    diffs = compare(gd, cd, floor_frac=1.0)
    mixed_form = {"x", "r32", "p32", "w32"}
    for name, d in diffs.items():
        assert d <= (1e-5 if name in mixed_form else 1e-10), (name, d)
    got, want = result_lines(gout, HEAT_KEYS), g["lines"]
    assert [words_and_counts(l) for l in got] == [words_and_counts(l) for l in want]
    assert_lines_close(got[:2], want[:2], 1e-9)


def test_heat_cg_converged_matches_reference(golden):
    """Both solvers to 1e-10 relative residual on 128^2: same iteration and
    refinement counts as the reference's sequential backend, checksums of the
    solutions within 1e-11."""
    g = golden["reference_runs"]["heat_cg_128"]
    gout, _ = run_app("heat_cg", "b200", g["args"])
    got = result_lines(gout, HEAT_KEYS)
    want = g["lines"]
    assert [words_and_counts(l) for l in got] == [words_and_counts(l) for l in want]
    for key in ("fp64 checksum", "mixed checksum"):
        a = [l for l in got if l.startswith(key)]
        b = [l for l in want if l.startswith(key)]
        assert_lines_close(a, b, 1e-11)
    rel = [float(l.split()[-1]) for l in got if l.startswith("fp64 it")][0]
    assert rel <= 1e-10


# further reference applications, built unchanged from the reference tree:
# (catalog name, arguments, dump comparison, text the application prints when
# its own check passes)
REF_APPS = [
    ("ref_lowdim", [], "exact", "All checks PASSED"),
    ("ref_multidim3d", [], "exact", "This run is considered PASSED"),
    ("ref_shsgc", [], "libm", "This run is considered PASSED"),
    ("ref_random", [], None, "This run is considered PASSED"),
    ("ref_compact", [], "roundoff", "Successful exit from OPS"),
    ("ref_adi_burger", [], "roundoff", "Successful exit from OPS"),
    ("ref_adi_burger3d", [], "roundoff", "Successful exit from OPS"),
    ("ref_tti", ["24", "20", "16"], "exact", "ops_NaNcheck_core called for ut0"),
    # half-precision dats (ACC<half>): IEEE binary16 arithmetic on both sides
    ("ref_halfprecision", [], "half", "This run is considered PASSED"),
    ("ref_lbm", [], "exact", "Test PASSED"),
    ("ref_tiling_fix", [], "exact", ""),
    # 4D blocks: par_loops over 4D ranges with ops_arg_idx, a 4D halo group
    ("ref_mblock4d", [], "exact", "Total Wall time"),
]


@pytest.mark.parametrize("name,args,mode,text", REF_APPS, ids=[a[0] for a in REF_APPS])
def test_more_reference_apps_match_oracle(tmp_path, name, args, mode, text):
    """Reference applications compiled unchanged by this backend's translator
    against the same applications on the CPU oracle: every dat (halos
    included) bit-exact ("exact"), or at round-off of the field's scale where
    the application solves tridiagonal systems ("roundoff": chunked PCR
    elimination order, 1e-12 of max|field|); the application's own pass
    message on the GPU run.  ref_random fills dats from a counter-based
    stream that differs from the CPU's by design, so only its own
    statistical check is asserted.  ref_shsgc's kernels call pow and sin,
    whose CUDA and glibc implementations may differ in the last ulp; its
    shock-capturing limiter amplifies that over the run ("libm": 1e-6 of the
    field's scale), and its own RMS check against the expected solution
    passes on the GPU."""
    import subprocess
    from tests.apprun import ensure
    dumps = {}
    outs = {}
    for fl in ("b200", "oracle"):
        exe = ensure(name, fl, shared=False)
        dumps[fl] = str(tmp_path / ("%s.dump" % fl))
        r = subprocess.run([exe, *args], cwd=str(tmp_path), capture_output=True, text=True,
                           env=dict(os.environ, OPS_DUMP_FILE=dumps[fl]), timeout=600)
        assert r.returncode == 0, (fl, r.stdout[-1500:], r.stderr[-1500:])
        outs[fl] = r.stdout
    assert text in outs["b200"], outs["b200"][-1500:]
    if mode == "exact":
        diffs = compare(dumps["b200"], dumps["oracle"])
        assert max(diffs.values()) == 0.0, {k: v for k, v in diffs.items() if v}
    elif mode == "roundoff":
        check_dumps(dumps["b200"], dumps["oracle"], tol=1e-12, float_tol=1e-6, floor_frac=1.0)
    elif mode == "libm":
        check_dumps(dumps["b200"], dumps["oracle"], tol=1e-6, float_tol=1e-5, floor_frac=1.0)
    elif mode == "half":
        # every binary16 operation is correctly rounded on both sides (the
        # host's _Float16 rounds each operation), so values agree; the
        # boundary values come from sin / exp in FP64 rounded to binary16,
        # where a last-ulp difference of libm may flip one rounding: at most
        # one binary16 ulp (2^-10 relative)
        diffs = compare(dumps["b200"], dumps["oracle"])
        assert max(diffs.values()) <= 2.0 ** -10, diffs


@pytest.mark.parametrize("solver", ["tl_use_jacobi", "tl_use_cg", "tl_use_chebyshev"])
def test_reference_tealeaf_known_answer_on_b200(solver):
    """TeaLeaf, written with the original OPS_ACCn kernel API, built unchanged:
    test problem 1 passes the reference's own check (within 0.001 % of the
    expected temperature)."""
    from tests.apprun import tealeaf_deck_test1
    d = tempfile.mkdtemp(prefix="tea_")
    with open(os.path.join(d, "tea.in"), "w") as f:
        f.write(tealeaf_deck_test1(solver))
    out = run_exe("ref_tealeaf", "b200", cwd=d)
    assert "This test is considered PASSED" in out, out[-1500:]


def test_reference_mgrid_known_answer_on_b200():
    """The reference's multigrid test (apps/c/mgrid, original OPS_ACCn kernels)
    built unchanged: a 6x6 field prolonged to 12x12 and 24x24 through prolong
    stencils (index / 2, with the +-1 neighbours) and restricted back through
    restrict stencils (index * 2), with periodic halo transfers in between;
    its own checks compare every point with the exact expected value and
    print PASSED."""
    out = run_exe("ref_mgrid", "b200", cwd=tempfile.mkdtemp(prefix="mgrid_"))
    assert "PASSED" in out and "FAILED" not in out, out[-1500:]


def test_reference_complex_on_b200():
    """The reference's complex test (apps/c/complex, OPS_ACCn kernels)
    built unchanged: a complexd dat filled with (x, y) from ops_arg_idx and
    an OPS_INC reduction of complexd values; its own check is the exact sum
    90 + 90i, and the dat written by ops_print_dat_to_txtfile holds the same
    values (the interior 6 x 6 points, in the reference's complex format)."""
    d = tempfile.mkdtemp(prefix="complex_")
    out = run_exe("ref_complex", "b200", cwd=d)
    assert "reduction result: 90+90i" in out and "PASSED" in out, out[-1500:]
    txt = open(os.path.join(d, "data.txt")).read().split("\n")
    rows = [l.split() for l in txt[1:] if l.strip()]
    # storage rows -2 .. 7 (halo depth 2); interior point (x, y) = x + y i
    for y in range(6):
        for x in range(6):
            assert rows[y + 2][x + 2] == "%.10f+%.10fi" % (x, y), (x, y, rows[y + 2][x + 2])


def test_reference_cpp_object_api_multidim_on_b200():
    """The reference's C++ object API test (apps/c/multiDim: OPS_instance
    created by the application with its own output stream, SoA storage set on
    the instance, instance->decl_* calls, block->decl_dat, halo_group->
    halo_transfer, reduction->get_result, globals whose length is a run-time
    value) built unchanged: its two-component reduction matches the expected
    value and it prints PASSED."""
    out = run_exe("ref_multidim_cpp", "b200", cwd=tempfile.mkdtemp(prefix="multidim_"))
    assert "This test is considered PASSED" in out, out[-1500:]
    assert "The test using ops_arg_gbl arguments passed!" in out


def test_reference_mb_trid_regression_on_b200():
    """The reference's mb_trid_test (C++ object API with `const char **argv`,
    two blocks, an ops_tridsolver_params per block, everything deleted again):
    a regression case for a crash in the reference; it must run to the end."""
    run_exe("ref_mb_trid", "b200", cwd=tempfile.mkdtemp(prefix="mbtrid_"))


def test_reference_mb_shsgc_on_b200():
    """The reference's mb_shsgc (shock-capturing shsgc written with the
    original OPS_ACCn kernel API, the Max_datatransfer variant) built
    unchanged: its own check of the post-shock error passes."""
    out = run_exe("ref_mb_shsgc", "b200", cwd=tempfile.mkdtemp(prefix="mbshsgc_"))
    assert "PASSED" in out, out[-1500:]


def test_reference_cloverleaf3d_known_answer_on_b200():
    """CloverLeaf 3D (original OPS_ACCn kernel API) built unchanged: test
    problem 2, 96^3 cells, 87 steps, passes the reference's own check."""
    from tests.apprun import clover3d_deck_test2
    d = tempfile.mkdtemp(prefix="clover3d_")
    with open(os.path.join(d, "clover.in"), "w") as f:
        f.write(clover3d_deck_test2())
    out = run_exe("ref_cloverleaf3d", "b200", cwd=d)
    assert "This test is considered PASSED" in out, out[-1500:]
