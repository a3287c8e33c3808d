"""Translator unit tests (CPU only): parsing, generated code, compilation."""

import os
import subprocess
import tempfile

import pytest

from ops_b200.translator.ops_translate import (Translator, find_calls, mask_comments_strings,
                                               parse_arg, parse_params, top_level_functions)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_mask_keeps_offsets():
    src = 'a(1) /* b(2) */ "c(3)" // d(4)\nx'
    m = mask_comments_strings(src)
    assert len(m) == len(src) and m.endswith("\nx") and "b(2)" not in m and "c(3)" not in m


def test_find_calls_nested_and_comments():
    src = ('ops_par_loop(k, "n", blk, 2, r, ops_arg_dat(d, 1, S, "double", OPS_READ), f(g(1), 2));'
           '\n// ops_par_loop(commented, x)\n')
    calls = find_calls(src, "ops_par_loop")
    assert len(calls) == 1
    args = calls[0][2]
    assert args[0] == "k" and args[5].startswith("ops_arg_dat") and args[6] == "f(g(1), 2)"


def test_parse_args_kinds():
    a = parse_arg('ops_arg_dat(u[i+ngrid*j], 1, S2D_00, "double", OPS_READ)', "t")
    assert (a.kind, a.ctype, a.dim, a.acc) == ("dat", "double", "1", "OPS_READ")
    a = parse_arg('ops_arg_dat_opt(o, 3, S, "float", OPS_WRITE, flag)', "t")
    assert a.kind == "dat" and a.opt and a.dim == "3"
    a = parse_arg('ops_arg_gbl(fields, NUM_FIELDS, "int", OPS_READ)', "t")
    assert (a.kind, a.dim) == ("gbl", "NUM_FIELDS")
    a = parse_arg('ops_arg_reduce(h, 2, "double", OPS_MIN)', "t")
    assert (a.kind, a.acc) == ("reduce", "OPS_MIN")
    assert parse_arg("ops_arg_idx()", "t").kind == "idx"
    with pytest.raises(SystemExit):
        parse_arg('ops_arg_gbl(x, 1, "double", OPS_INC)', "t")


def test_parse_params():
    ps = parse_params("const ACC<double> &u, ACC<float>& v, const int *idx, double* r")
    assert [p.is_acc for p in ps] == [True, True, False, False]
    assert [p.base_type for p in ps] == ["double", "float", "int", "double"]


def test_top_level_functions_skip_structs_and_comments():
    text = ("#include \"x.h\"\nstruct S { int a; };\n"
            "void k1(const ACC<double> &u /* note */, double *r) { *r += u(0,0); }\n"
            "static inline double helper(double a) { return a * 2; }\n")
    fs = {f.name: f for f in top_level_functions(text, "h")}
    assert set(fs) == {"k1", "helper"}
    assert fs["k1"].params is not None and len(fs["k1"].params) == 2


def test_translate_and_compile_opsunit():
    out = tempfile.mkdtemp(prefix="tr_")
    src = os.path.join(ROOT, "apps", "opsunit", "opsunit.cpp")
    Translator([src], [], "opsunit", out).run()
    cu = open(os.path.join(out, "opsunit_kernels.cu")).read()
    # one kernel per loop signature, both aliasing variants, restrict pointers
    for k in ("ou_fill", "ou_vec", "ou_stencil", "ou_strided", "ou_reduce", "ou_opt", "ou_rw",
              "ou_colsum"):
        assert "ob2k_%s(" % k in cu
        assert "ob2i_%s_R" % k in cu and "ob2i_%s_A" % k in cu
    assert "__restrict__" in cu and "__constant__ double ou_scale;" in cu
    assert "ob2::final_combine<double, OPS_MIN>" in cu
    # the kernels' divisions go through ob2::div (compiled below), unless
    # OPS_B200_DDIV=0 at translation time
    assert "::ob2::div(" in cu and "1 as ob2::div, 0 kept as written" in cu
    out0 = tempfile.mkdtemp(prefix="tr0_")
    os.environ["OPS_B200_DDIV"] = "0"
    try:
        Translator([src], [], "opsunit", out0).run()
    finally:
        del os.environ["OPS_B200_DDIV"]
    cu0 = open(os.path.join(out0, "opsunit_kernels.cu")).read()
    assert "::ob2::div(" not in cu0 and "all kept as written (OPS_B200_DDIV=0)" in cu0
    ops = open(os.path.join(out, "opsunit_ops.cpp")).read()
    assert "ops_par_loop(" not in ops.replace("ops_par_loop_", "")
    # compile the kernels for sm_100a (cross-compiles without a GPU)
    nvcc = "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not present")
    r = subprocess.run([nvcc, "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-w",
                        "--fmad=false", "-I" + os.path.join(ROOT, "include"),
                        "-I" + os.path.join(ROOT, "apps", "opsunit"), "-c",
                        os.path.join(out, "opsunit_kernels.cu"), "-o",
                        os.path.join(out, "k.o")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


def test_prolong_stencil_arguments_divide_the_loop_index():
    """A dat argument whose stencil variable comes from ops_decl_prolong_stencil
    reads its dat at the loop index divided by the multigrid stride
    (ops_translator/resources/templates/cpp/mpi_openmp/loop_host.cpp.j2:83-89);
    the stub marks it for the runtime, and other arguments keep plain
    indexing."""
    d = tempfile.mkdtemp(prefix="ob2_prolong_")
    src = os.path.join(d, "mg.cpp")
    with open(os.path.join(d, "mg_kernels.h"), "w") as f:
        f.write("void copy_k(const ACC<double> &c, ACC<double> &f) { f(0, 0) = c(0, 0); }\n")
    with open(src, "w") as f:
        f.write('#define OPS_2D\n#include "ops_seq_v2.h"\n#include "mg_kernels.h"\n'
                "int main(int argc, char **argv) {\n"
                "  ops_init(argc, argv, 1);\n"
                '  ops_block g = ops_decl_block(2, "g");\n'
                "  int s00[] = {0, 0}, st[] = {2, 2};\n"
                '  ops_stencil S00 = ops_decl_stencil(2, 1, s00, "00");\n'
                '  ops_stencil SP = ops_decl_prolong_stencil(2, 1, s00, st, "p");\n'
                "  ops_dat c = 0, fi = 0; int r[] = {0, 8, 0, 8};\n"
                '  ops_par_loop(copy_k, "copy_k", g, 2, r, ops_arg_dat(c, 1, SP, "double", OPS_READ),\n'
                '               ops_arg_dat(fi, 1, S00, "double", OPS_WRITE));\n'
                '  ops_par_loop(copy_k, "copy_k", g, 2, r, ops_arg_dat(c, 1, S00, "double", OPS_READ),\n'
                '               ops_arg_dat(fi, 1, S00, "double", OPS_WRITE));\n'
                "  ops_exit();\n}\n")
    out = os.path.join(d, "gen")
    Translator([src], [d], "mg", out).run()
    cu = open(os.path.join(out, "mg_kernels.cu")).read()
    # two loops: one with the prolong argument (mask bit 0), one without
    assert cu.count("L.prolong_mask = 1u;") == 1 and cu.count("L.prolong_mask = 0u;") == 1
    assert "(x / p.mx0)" in cu and "p.mx0 = arg0.stencil->mgrid_stride[0];" in cu
    assert "(x / p.mx1)" not in cu


def test_cpp_api_constants_and_runtime_length_globals():
    """Constants declared through the C++ object API (instance->decl_const)
    become device constants like ops_decl_const ones; an ops_arg_gbl whose
    length is a run-time variable gets a fixed-capacity slot in the parameter
    block (the stub rejects longer arrays), one with a literal or macro
    length keeps that length."""
    d = tempfile.mkdtemp(prefix="ob2_cppapi_")
    src = os.path.join(d, "c.cpp")
    with open(os.path.join(d, "c_kernels.h"), "w") as f:
        f.write("void k(ACC<double> &u, const double *a, const double *b) {"
                " u(0, 0) = a[0] + b[0] + kc; }\n")
    with open(src, "w") as f:
        f.write('#define OPS_2D\n#define OPS_CPP_API\n#include "ops_seq_v2.h"\n'
                "int kc = 3;\n#define NB 4\n"
                '#include "c_kernels.h"\n'
                "int main(int argc, char **argv) {\n"
                "  OPS_instance *instance = new OPS_instance(argc, argv, 1);\n"
                '  instance->decl_const("kc", 1, "int", &kc);\n'
                "  ops_block g = 0; ops_dat u = 0; ops_stencil S = 0; int n = 5;\n"
                "  double a[5], b[NB]; int r[] = {0, 4, 0, 4};\n"
                '  ops_par_loop(k, "k", g, 2, r, ops_arg_dat(u, 1, S, "double", OPS_WRITE),\n'
                '               ops_arg_gbl(a, n, "double", OPS_READ),\n'
                '               ops_arg_gbl(b, NB, "double", OPS_READ));\n'
                "  delete instance;\n}\n")
    out = os.path.join(d, "gen")
    Translator([src], [d], "c", out).run()
    cu = open(os.path.join(out, "c_kernels.cu")).read()
    assert "__constant__ int kc;" in cu
    assert "double g1[64];" in cu and "double g2[NB];" in cu


def test_fused_dispatcher_ids_name_each_loops_own_body():
    """Every stub that offers its loop to the fused dispatcher (ob2fk) names
    an id whose `case` runs that loop's own body on that loop's parameter
    block; an id pointing at another loop's body would run it on the wrong
    parameters."""
    import re
    out = tempfile.mkdtemp(prefix="tr_fuse_")
    src = os.path.join(ROOT, "apps", "opsunit", "opsunit.cpp")
    Translator([src], [], "opsunit", out).run()
    cu = open(os.path.join(out, "opsunit_kernels.cu")).read()
    cases = {int(k): (body, prm) for k, body, prm in
             re.findall(r"case (\d+): (ob2b_\w+)<false, IDX32>\(\*\(const (\w+) \*\)prm", cu)}
    stubs = re.findall(r"void (ops_par_loop_\w+)\(.*?\n\}\n", cu, flags=re.S)
    ids = {}
    for m in re.finditer(r"void ops_par_loop_(\w+)\((.*?)\n\}\n", cu, flags=re.S):
        f = re.search(r"L\.fuse_id = (\d+);", m.group(2))
        if f:
            ids[m.group(1)] = int(f.group(1))
    assert stubs and ids and len(set(ids.values())) == len(ids)
    for name, k in ids.items():
        assert k in cases, (name, k)
        assert cases[k][0] == "ob2b_" + name and cases[k][1].startswith("ob2p_"), (name, cases[k])


DIV_CASES = [
    "a * b / c", "a / b * c", "-a / b", "a / -b", "a + b * c / d - e", "a / b / c",
    "(double)i / n", "f1(a) / (b + c)", "MIN(a / b, c)", "SIGN(a / b, c)", "a / SQ(b)",
    "BAD / c", "K / c", "p->x / s.y[1]", "c > 0 ? a / b : d / e", "*q / 2", "0.5*(a-b)/c",
    "a /* note */ / b", "(double)(a) / b", "-a * b / c / d * e", "a * -b / c", "d / 3",
    "i / j * a", "a / i / j", "2 * a / 3.0 + b / -c", "(a + b) / (c - d) / e",
    "SCALE(a / b)", "MAX(a / b, c / d) / e",
]


def test_division_rewrite_keeps_the_grouping():
    """Every rewritten expression, with ob2::div defined as the operator
    itself, evaluates to the same bits as the original on random values: the
    rewrite chose the operands C's grammar gives each `/` (a wrong grouping
    changes the rounding, or the integer quotient, on almost every sample)."""
    from ops_b200.translator.divrewrite import macro_table, rewrite_divisions
    macros = macro_table([open(os.path.join(ROOT, "include", "ops_lib_core.h")).read(),
                          "#define SQ(x) x*x\n#define K 3.0\n#define BAD a+b\n"
                          "#define SCALE(v) 2.0*v\n"])
    rewritten = []
    n_done = 0
    for e in DIV_CASES:
        r, done, _ = rewrite_divisions("{ return " + e + "; }", mask_comments_strings, macros)
        n_done += done
        rewritten.append(r[len("{ return "):-len("; }")])
    assert rewritten[0] == "::ob2::div(a * b, c)" and rewritten[1] == "::ob2::div(a, b) * c"
    assert rewritten[10] == "a / SQ(b)" and rewritten[11] == "BAD / c"  # unsafe macros kept
    assert rewritten[18] == "(double)(a) / b"  # a cast of a group is not parsed: kept
    # SCALE puts its argument after a `*`: a division passed to it is kept
    assert rewritten[26] == "SCALE(a / b)"
    assert rewritten[27] == "::ob2::div(MAX(::ob2::div(a, b), ::ob2::div(c, d)), e)"
    for kept in ("sizeof x / y", "++i / 2", "--i / 2", "sizeof(double) / 2"):
        r, done, _ = rewrite_divisions("{ " + kept + "; }", mask_comments_strings, macros)
        assert done == 0 and r == "{ " + kept + "; }", r
    assert n_done >= 29
    src = ["#include <cstdio>", "#include <cstring>", "#include <cstdlib>",
           '#include "ops_lib_core.h"',
           "namespace ob2 { template <class A, class B> auto div(A a, B b) { return a / b; } }",
           "#define SQ(x) x*x", "#define K 3.0", "#define BAD a+b", "#define SCALE(v) 2.0*v",
           "struct P { double x; double y[2]; };",
           "static double f1(double v) { return v * 1.5; }"]
    args = "double a, double b, double c, double d, double e, int i, int j, int n, P *p, P s, double *q"
    for k, (o, r) in enumerate(zip(DIV_CASES, rewritten)):
        src.append("static double o%d(%s) { return %s; }" % (k, args, o))
        src.append("static double r%d(%s) { return %s; }" % (k, args, r))
    src.append("int main() { srand(7); int bad = 0;")
    src.append(" for (int t = 0; t < 20000; t++) {")
    src.append("  double v[5]; for (int m = 0; m < 5; m++) v[m] = (rand() - RAND_MAX / 2) /"
               " (double)(rand() % 997 + 1) + 1e-3;")
    src.append("  int i = rand() % 200 - 100, j = rand() % 13 + 1, n = rand() % 50 + 1;")
    src.append("  P pp = {v[1] * 3.7, {v[2] * 0.3, v[3] * 1.9}}; double qq = v[4] * 7.1;")
    for k in range(len(DIV_CASES)):
        src.append("  { double x = o%d(v[0], v[1], v[2], v[3], v[4], i, j, n, &pp, pp, &qq),"
                   " y = r%d(v[0], v[1], v[2], v[3], v[4], i, j, n, &pp, pp, &qq);"
                   " if (memcmp(&x, &y, 8)) { if (bad < 5) printf(\"case %d\\n\"); bad++; } }"
                   % (k, k, k))
    src.append(" }")
    src.append(" printf(\"bad %d\\n\", bad); return bad != 0; }")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.cpp")
        open(c, "w").write("\n".join(src) + "\n")
        exe = os.path.join(d, "t")
        subprocess.run(["g++", "-std=c++17", "-O1", "-ffp-contract=off", "-I",
                        os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        r = subprocess.run([exe], capture_output=True, text=True)
        assert r.returncode == 0, r.stdout


def test_markstein_division_steps_round_correctly_on_the_host():
    """The steps of ob2::ddiv (include/ops_b200_kernel.h) restated on the
    host with a poorer start than the GPU's (the float reciprocal, about 24
    bits, in place of rcp.approx.ftz.f64): three Newton-Raphson steps on the
    reciprocal, then Markstein's quotient correction, all with fused
    multiply-adds, equal the IEEE quotient on random operands of the fast
    domain (both in [2^-500, 2^500)), near-midpoint quotients and zero
    numerators.  The GPU test (tests/test_gpu_ddiv.py) checks the device
    code itself against CUDA's `/`."""
    src = r'''
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
static uint64_t st = 88172645463325252ull;
static uint64_t rnd() { st ^= st << 13; st ^= st >> 7; st ^= st << 17; return st; }
static double with_exp(uint64_t bits, unsigned e) {
  bits = (bits & 0x800fffffffffffffull) | ((uint64_t)e << 52);
  double d; memcpy(&d, &bits, 8); return d;
}
static double ddiv(double a, double b) {
  double y = (double)(1.0f / (float)b);
  double e = std::fma(-b, y, 1.0); y = std::fma(y, e, y);
  e = std::fma(-b, y, 1.0); y = std::fma(y, e, y);
  e = std::fma(-b, y, 1.0); y = std::fma(y, e, y);
  const double q0 = a * y, r = std::fma(-b, q0, a);
  return a == 0.0 ? q0 : std::fma(r, y, q0);
}
int main() {
  long bad = 0, n = 0;
  for (int mode = 0; mode < 3; mode++)
    for (int t = 0; t < 2000000; t++) {
      double a, b;
      const uint64_t r0 = rnd(), r1 = rnd(), r2 = rnd();
      b = with_exp(r1, 1023 - 100 + (unsigned)(r2 % 200));
      if ((r1 & 0xfffffffffffffull) == 0xfffffffffffffull) continue;  // all-ones: IEEE path
      if (mode == 0) a = with_exp(r0, 523 + (unsigned)((r2 >> 20) % 1000));
      else if (mode == 1) {
        const double q = std::fabs(with_exp(r0, 1023 + (unsigned)((r2 >> 20) % 64) - 32));
        a = std::fma(b, q, b * std::ldexp(std::fabs(q), -53));  // q + half an ulp, times b
      } else a = (r0 & 1) ? -0.0 : 0.0;
      const double want = a / b, got = ddiv(a, b);
      n++;
      if (memcmp(&want, &got, 8)) { if (bad < 3) printf("%a / %a: %a vs %a\n", a, b, got, want); bad++; }
    }
  printf("%ld of %ld differ\n", bad, n);
  return bad != 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "m.cpp")
        open(c, "w").write(src)
        exe = os.path.join(d, "m")
        subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-mfma", c, "-o", exe],
                       check=True)
        r = subprocess.run([exe], capture_output=True, text=True)
        assert r.returncode == 0, r.stdout
