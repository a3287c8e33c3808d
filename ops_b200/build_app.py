"""Build an OPS application for the B200 backend.

    python -m ops_b200.build_app --app NAME --out DIR [-I dir ...] [--shared]
                                 [--define X] src1.cpp src2.cpp ...

Steps: run the translator (ops_b200/translator), compile the generated
kernels file with nvcc for sm_100a, compile the rewritten sources, and link
against libops_b200.so (rpath set, so the result runs in place).  With
--shared the app is linked as a shared library whose ``main`` is renamed to
``ops_app_main`` so that a caller (tests, bench) can load it with ctypes and
run it in-process.

Replaces the per-app build recipes of the reference
(makefiles/Makefile.c_app_legacy:143-247, cuda target).
"""

from __future__ import annotations

import argparse
import os
import shlex
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(HERE, "lib")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

sys.path.insert(0, ROOT)
from ops_b200.translator.ops_translate import Translator  # noqa: E402


def run(cmd, verbose):
    if verbose:
        print("+", " ".join(shlex.quote(c) for c in cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise SystemExit("build step failed: %s" % cmd[0])
    return r


def ensure_lib(verbose=False):
    lib = os.path.join(LIBDIR, "libops_b200.so")
    run(["make", "-s", "-C", HERE, "-j8"], verbose)
    return lib


def build(app, out, sources, incs, defines=(), shared=False, verbose=False, jobs=8,
          extra_nvcc=(), rename_main=None):
    """rename_main: {source basename: new name} renames that source's main
    (used by harnesses that drive an app's functions themselves)."""
    ensure_lib(verbose)
    os.makedirs(out, exist_ok=True)
    gen = os.path.join(out, "gen")
    srcs = [os.path.abspath(s) for s in sources]
    incs = [os.path.abspath(i) for i in incs]
    Translator(srcs, incs, app, gen).run()
    common = ["-I" + INCLUDE] + ["-I" + i for i in incs] + ["-D" + d for d in defines]
    common += ["-I" + os.path.dirname(s) for s in srcs]
    objs = []
    procs = []
    cu = os.path.join(gen, app + "_kernels.cu")
    cu_o = os.path.join(out, app + "_kernels.o")
    # IEEE arithmetic by default (no FMA contraction), as the reference's
    # IEEE build (makefiles/Makefile.cuda:55-56): the generated kernels then
    # round exactly like the host code of the same user kernels.
    if os.environ.get("OPS_B200_FMAD", "0") != "1":
        extra_nvcc = ("--fmad=false",) + tuple(extra_nvcc)
    procs.append((subprocess.Popen(
        [NVCC, "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC",
         "--expt-relaxed-constexpr", "-w", *extra_nvcc, *common, "-c", cu, "-o", cu_o],
        stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True), cu))
    objs.append(cu_o)
    for s in srcs:
        base = os.path.splitext(os.path.basename(s))[0]
        g = os.path.join(gen, base + "_ops.cpp")
        o = os.path.join(out, base + "_ops.o")
        cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-w", *common,
               "-I" + os.path.join(CUDA, "include"), "-c", g, "-o", o]
        if rename_main and os.path.basename(s) in rename_main:
            cmd.insert(1, "-Dmain=" + rename_main[os.path.basename(s)])
        elif shared and not rename_main:
            cmd.insert(1, "-Dmain=ops_app_main")
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                                       text=True), g))
        objs.append(o)
        while len([p for p, _ in procs if p.poll() is None]) >= jobs:
            procs[0][0].wait()
    failed = False
    for p, name in procs:
        outp, _ = p.communicate()
        if p.returncode != 0:
            sys.stderr.write("---- %s\n%s\n" % (name, outp))
            failed = True
    if failed:
        raise SystemExit("compilation failed")
    target = os.path.join(out, ("lib%s.so" % app) if shared else app)
    link = [NVCC, *ARCH, "-o", target, *objs, "-L" + LIBDIR, "-lops_b200",
            "-Xlinker", "-rpath=" + LIBDIR, "-L" + os.path.join(CUDA, "lib64"), "-lcudart"]
    if shared:
        # -Bsymbolic: the app's own globals must bind inside the library
        # (glibc exports names such as `step` that would interpose them)
        link[1:1] = ["-shared", "-Xlinker", "-Bsymbolic"]
    run(link, verbose)
    return target


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("sources", nargs="+")
    ap.add_argument("--app", required=True)
    ap.add_argument("--out", required=True)
    ap.add_argument("-I", dest="incs", action="append", default=[])
    ap.add_argument("-D", "--define", dest="defines", action="append", default=[])
    ap.add_argument("--shared", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    t = build(a.app, a.out, a.sources, a.incs, a.defines, a.shared, a.verbose)
    print(t)
    return 0


if __name__ == "__main__":
    sys.exit(main())
