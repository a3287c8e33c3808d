"""Catalogue of the OPS applications used by the tests and the benchmark, and
how to build each one in every flavour.

Flavours
  b200     this backend: translator + libops_b200.so (sm_100a)
  oracle   the CPU oracle: oracle/include/ops_seq_v2.h + liboracle_ops.so
  ref_seq  the reference's own sequential backend (ops_seq_v2.h + libops_seq.a)
  ref_omp  the reference's own OpenMP backend (legacy translator + libops_seq.a)
  ref_cuda the reference's own CUDA backend (legacy translator's CUDA kernels +
           libops_cuda.a, sm_100): a same-machine measure of the reference's GPU
           code, reported as context

Applications are either this repository's drivers under apps/ (our code, on the
unchanged OPS API) or reference applications, whose sources are read from the
reference tree named by OPS_REFERENCE_TREE at build time only (without it,
only the prebuilt binaries are used).  Product builds (the b200 flavour) of
reference applications go under apps/_build/ref/; the checker builds (the
oracle flavour and every ref_* flavour) go under oracle/_ref/.  Both are
git-ignored; the built binaries travel to the GPU machine, the sources do not.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

# the upstream OPS tree, read at build time only; unset: nothing is rebuilt
# from it, and the reference-derived builds already present are used as they are
REF = os.environ.get("OPS_REFERENCE_TREE", "")
_REF_ROOT = REF or os.path.join(os.sep, "nonexistent-ops-reference-tree")
ORACLE_LIB_DIR = os.path.join(ROOT, "oracle", "_build")
REF_OUT = os.path.join(ROOT, "oracle", "_ref")

CLOVER_SRCS = ["clover_leaf.cpp", "initialise_chunk.cpp", "generate.cpp", "ideal_gas.cpp",
               "update_halo.cpp", "field_summary.cpp", "viscosity.cpp", "calc_dt.cpp", "PdV.cpp",
               "revert.cpp", "accelerate.cpp", "flux_calc.cpp", "advec_cell.cpp",
               "advec_mom.cpp", "reset_field.cpp", "start.cpp", "time_step.cpp",
               "build_field.cpp", "read_input.cpp", "initialise.cpp", "advection.cpp"]

TEALEAF_SRCS = ["tea_leaf.cpp", "field_summary.cpp", "generate.cpp", "initialise_chunk.cpp",
                "start.cpp", "set_field.cpp", "tea_leaf_cg.cpp", "tea_leaf_cheby.cpp",
                "tea_leaf_common.cpp", "tea_leaf_jacobi.cpp", "tea_leaf_ppcg.cpp",
                "update_halo.cpp", "build_field.cpp", "diffuse.cpp", "initialise.cpp",
                "read_input.cpp", "tea_solve.cpp", "timestep.cpp"]
CLOVER3D_SRCS = ["clover_leaf.cpp", "initialise_chunk.cpp", "generate.cpp", "ideal_gas.cpp",
                 "update_halo.cpp", "field_summary.cpp", "viscosity.cpp", "calc_dt.cpp",
                 "PdV.cpp", "revert.cpp", "accelerate.cpp", "flux_calc.cpp", "advec_cell.cpp",
                 "advec_mom.cpp", "reset_field.cpp", "start.cpp", "time_step.cpp",
                 "build_field.cpp", "read_input.cpp", "initialise.cpp", "advection.cpp"]

# name -> (kind, source dir, sources, translated sources (legacy translator))
APPS = {
    "poisson_mb": ("own", os.path.join(ROOT, "apps", "poisson_mb"), ["poisson_mb.cpp"], None),
    "adi3d": ("own", os.path.join(ROOT, "apps", "adi3d"), ["adi3d.cpp"], None),
    "heat_cg": ("own", os.path.join(ROOT, "apps", "heat_cg"), ["heat_cg.cpp"], None),
    "opsunit": ("own", os.path.join(ROOT, "apps", "opsunit"), ["opsunit.cpp"], None),
    "hdunit": ("own", os.path.join(ROOT, "apps", "hdunit"), ["hdunit.cpp"], None),
    "ref_poisson": ("ref", os.path.join(_REF_ROOT, "apps", "c", "poisson"), ["poisson.cpp"], None),
    "ref_mblock": ("ref", os.path.join(_REF_ROOT, "apps", "c", "mblock"), ["mblock.cpp"], None),
    # 4D blocks: two 4^4 blocks filled from ops_arg_idx, joined by a 4D halo
    "ref_mblock4d": ("ref", os.path.join(_REF_ROOT, "apps", "c", "mblock4D"), ["mblock.cpp"], None),
    "ref_laplace": ("ref", os.path.join(_REF_ROOT, "apps", "c", "laplace2d_tutorial", "step7"),
                    ["laplace2d.cpp"], None),
    # further reference applications, built unchanged (the v2 ACC API)
    "ref_lowdim": ("ref", os.path.join(_REF_ROOT, "apps", "c", "lowdim_test"), ["lowdim.cpp"], None),
    "ref_multidim3d": ("ref", os.path.join(_REF_ROOT, "apps", "c", "multiDim3D"), ["multidim.cpp"],
                       None),
    "ref_shsgc": ("ref", os.path.join(_REF_ROOT, "apps", "c", "shsgc"), ["shsgc.cpp"], None),
    "ref_compact": ("ref", os.path.join(_REF_ROOT, "apps", "c", "compact_scheme"),
                    ["compact_scheme.cpp"], None),
    "ref_random": ("ref", os.path.join(_REF_ROOT, "apps", "c", "random"), ["random.cpp"], None),
    "ref_tiling_fix": ("ref", os.path.join(_REF_ROOT, "apps", "c", "tiling_fix"), ["minisenga.cpp"],
                       None),
    "ref_adi_burger": ("ref", os.path.join(_REF_ROOT, "apps", "c", "adi_burger"), ["adi_burger.cpp"],
                       None),
    "ref_adi_burger3d": ("ref", os.path.join(_REF_ROOT, "apps", "c", "adi_burger_3D"),
                         ["adi_burger_3D.cpp"], None),
    "ref_tti": ("ref", os.path.join(_REF_ROOT, "apps", "c", "tti"), ["tti.cpp"], None),
    # half-precision dats (ACC<half>): Jacobi on a 4094^2 grid in binary16
    "ref_halfprecision": ("ref", os.path.join(_REF_ROOT, "apps", "c", "halfprecision"),
                          ["laplace2d.cpp"], None),
    # multi-block shsgc (halo transfers between the blocks every step)
    "ref_mb_shsgc": ("ref", os.path.join(_REF_ROOT, "apps", "c", "mb_shsgc", "Max_datatransfer"),
                     ["shsgc.cpp"], None),
    # the lattice-Boltzmann tutorial app (final step), the OpenSBLI wave test
    "ref_lbm": ("ref", os.path.join(_REF_ROOT, "apps", "c", "ops-lbm", "step5"),
                ["lattboltz2d.cpp"], None),
    "ref_wave": ("ref", os.path.join(_REF_ROOT, "apps", "c", "wave_test"), ["opensbli.cpp"], None),
    # reference applications written with the original OPS_ACCn kernel API
    # (b200 flavour only: the oracle restates the ACC<> API)
    "ref_tealeaf": ("ref", os.path.join(_REF_ROOT, "apps", "c", "TeaLeaf"), TEALEAF_SRCS, None),
    "ref_mgrid": ("ref", os.path.join(_REF_ROOT, "apps", "c", "mgrid"), ["mgrid.cpp"], None),
    # complexd dats and an OPS_INC reduction of complexd values
    "ref_complex": ("ref", os.path.join(_REF_ROOT, "apps", "c", "complex"), ["complex.cpp"], None),
    # the reference's C++ object API test (OPS_CPP_API: OPS_instance methods)
    "ref_multidim_cpp": ("ref", os.path.join(_REF_ROOT, "apps", "c", "multiDim"), ["multidim.cpp"],
                         None),
    "ref_mb_trid": ("ref", os.path.join(_REF_ROOT, "apps", "c", "mb_trid_test"), ["mb_trid.cpp"], None),
    "ref_cloverleaf3d": ("ref", os.path.join(_REF_ROOT, "apps", "c", "CloverLeaf_3D"), CLOVER3D_SRCS,
                         None),
    "cloverleaf": ("ref", os.path.join(_REF_ROOT, "apps", "c", "CloverLeaf"), CLOVER_SRCS,
                   CLOVER_SRCS[:15]),
    # the CloverLeaf step harness: the CloverLeaf sources plus apps/clover_step
    "clover_step": ("mixed", os.path.join(_REF_ROOT, "apps", "c", "CloverLeaf"), CLOVER_SRCS,
                    CLOVER_SRCS[:15]),
}
CLOVER_STEP_SRC = os.path.join(ROOT, "apps", "clover_step", "clover_step.cpp")
# shared headers of this repository's drivers and harnesses (apps/dumpdats.h)
APPS_DIR = os.path.join(ROOT, "apps")


def build_dir(name: str, flavour: str) -> str:
    kind = APPS[name][0]
    if kind == "own" and not flavour.startswith("ref_"):
        return os.path.join(ROOT, "apps", name, "_build", flavour)
    if flavour == "b200":  # product build of a reference application
        return os.path.join(ROOT, "apps", "_build", "ref", name, flavour)
    return os.path.join(REF_OUT, "apps", name, flavour)


def artifact(name: str, flavour: str, shared: bool = False) -> str:
    d = build_dir(name, flavour)
    return os.path.join(d, ("lib%s.so" % name) if shared else name)


def _run(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout[-4000:] + r.stderr[-8000:])
        raise RuntimeError("build step failed: %s" % " ".join(cmd[:3]))
    return r


def sources_of(name: str):
    kind, d, srcs, _ = APPS[name]
    paths = [os.path.join(d, s) for s in srcs]
    if name == "clover_step":
        paths.append(CLOVER_STEP_SRC)
    return d, paths


def available(name: str) -> bool:
    d, paths = sources_of(name)
    return all(os.path.isfile(p) for p in paths)


def ensure_oracle_lib() -> str:
    _run(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    return os.path.join(ORACLE_LIB_DIR, "liboracle_ops.so")


def ensure_ref_lib() -> str:
    if not REF or not os.path.isdir(REF):
        lib = os.path.join(REF_OUT, "lib", "libops_seq.a")
        if os.path.exists(lib):
            return lib
        raise RuntimeError("reference tree not present (set OPS_REFERENCE_TREE)")
    _run(["make", "-s", "-C", os.path.join(ROOT, "oracle", "ref"), "lib", "-j8", "REF=" + REF])
    return os.path.join(REF_OUT, "lib", "libops_seq.a")


CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
# the reference's default CUDA flags (makefiles/Makefile.cuda:15-18) for sm_100
REF_NVCCFLAGS = ["-Xcompiler=-fPIC", "-O3", "-g", "-std=c++14",
                 "-gencode", "arch=compute_100,code=sm_100", "-w"]


def ensure_ref_cuda_lib() -> str:
    """The reference's own CUDA backend (libops_cuda.a, oracle/ref/Makefile
    cudalib): a same-machine measure of the reference's GPU code."""
    lib = os.path.join(REF_OUT, "lib", "libops_cuda.a")
    if not REF or not os.path.isdir(REF):
        if os.path.exists(lib):
            return lib
        raise RuntimeError("reference tree not present (set OPS_REFERENCE_TREE)")
    _run(["make", "-s", "-C", os.path.join(ROOT, "oracle", "ref"), "cudalib", "-j8",
          "REF=" + REF])
    return lib


def _deps(name: str, flavour: str):
    d, paths = sources_of(name)
    deps = list(paths)
    for dd in {d, os.path.dirname(CLOVER_STEP_SRC) if name == "clover_step" else d}:
        if os.path.isdir(dd):
            deps += [os.path.join(dd, f) for f in os.listdir(dd) if f.endswith(".h")]
    if flavour == "b200":
        deps.append(os.path.join(ROOT, "ops_b200", "translator", "ops_translate.py"))
        deps.append(os.path.join(ROOT, "ops_b200", "translator", "divrewrite.py"))
        deps.append(os.path.join(ROOT, "ops_b200", "build_app.py"))
        inc = os.path.join(ROOT, "include")
        deps += [os.path.join(inc, f) for f in os.listdir(inc)]
    elif flavour == "oracle":
        deps += [os.path.join(ROOT, "oracle", "include", "ops_seq_v2.h"),
                 os.path.join(ROOT, "include", "ops_lib_core.h")]
    return [p for p in deps if os.path.exists(p)]


def stale(name: str, flavour: str, shared: bool = False) -> bool:
    target = artifact(name, flavour, shared)
    if not os.path.exists(target):
        return True
    if not available(name):
        return False  # prebuilt and no sources to rebuild from
    if flavour.startswith("ref_") and not REF:
        return False  # prebuilt against the reference tree, which is not named
    t = os.path.getmtime(target)
    return any(os.path.getmtime(p) > t for p in _deps(name, flavour))


def build(name: str, flavour: str, shared: bool = False, force: bool = False) -> str:
    """Build one application flavour (when missing or older than its
    sources, headers or the translator); returns the executable / library."""
    out = build_dir(name, flavour)
    target = artifact(name, flavour, shared)
    if not force and not stale(name, flavour, shared):
        return target
    d, paths = sources_of(name)
    os.makedirs(out, exist_ok=True)
    extra_defs = []
    if name == "clover_step":
        extra_defs = ["-Dmain=clover_leaf_main"]
    if flavour == "b200":
        from ops_b200.build_app import build as b200_build
        defs = [x[2:] for x in extra_defs]
        if name == "clover_step":
            # only clover_leaf.cpp's main is renamed; the harness keeps its own
            return _build_b200_clover_step(out, d, paths, shared)
        return b200_build(name, out, paths, [d, APPS_DIR], defines=defs, shared=shared)
    if flavour == "oracle":
        lib = ensure_oracle_lib()
        inc = ["-I" + os.path.join(ROOT, "oracle", "include"), "-I" + os.path.join(ROOT, "include"),
               "-I" + d, "-I" + APPS_DIR]
        objs = []
        for p in paths:
            o = os.path.join(out, os.path.basename(p) + ".o")
            # binary16 (`half`) arithmetic rounded after every operation, as
            # CUDA's __half does (GCC would otherwise evaluate it in float)
            cmd = ["g++", "-O2", "-g", "-std=c++17", "-fPIC", "-w", "-fexcess-precision=16", *inc]
            if name == "clover_step" and os.path.basename(p) == "clover_leaf.cpp":
                cmd += extra_defs
            if shared and name != "clover_step":
                cmd += ["-Dmain=ops_app_main"]
            _run(cmd + ["-c", p, "-o", o])
            objs.append(o)
        link = ["g++", "-o", target, *objs, "-L" + ORACLE_LIB_DIR, "-loracle_ops",
                "-Wl,-rpath," + ORACLE_LIB_DIR]
        if shared:
            link[1:1] = ["-shared", "-Wl,-Bsymbolic"]
        _run(link)
        return target
    if flavour in ("ref_seq", "ref_omp", "ref_cuda"):
        lib = ensure_ref_lib()
        if flavour == "ref_cuda":
            lib = ensure_ref_cuda_lib()
        rinc = os.path.join(REF, "ops", "c", "include")
        srcdir = os.path.join(out, "src")
        if os.path.isdir(srcdir):
            shutil.rmtree(srcdir)
        os.makedirs(srcdir)
        for f in os.listdir(d):
            if f.endswith((".cpp", ".h", ".in")):
                shutil.copy(os.path.join(d, f), srcdir)
        objs_src = [os.path.join(srcdir, os.path.basename(p)) for p in paths
                    if p != CLOVER_STEP_SRC]
        flags = ["-O3", "-std=c++14", "-fPIC", "-w", "-fopenmp", "-Dgnu", "-I" + rinc, "-I" + srcdir,
                 "-I" + APPS_DIR]
        pre_objs = []
        if flavour in ("ref_omp", "ref_cuda"):
            trans = APPS[name][3] or APPS[name][2]
            _run([sys.executable, os.path.join(REF, "ops_translator_legacy", "c", "ops.py"),
                  *trans], cwd=srcdir)
            objs_src = [os.path.join(srcdir, (s[:-4] + "_ops.cpp") if s in trans else s)
                        for s in APPS[name][2]]
            if flavour == "ref_omp":
                objs_src.append(os.path.join(srcdir, "mpi_openmp", "mpi_openmp_kernels.cpp"))
            else:  # the legacy translator's CUDA kernels (Makefile.c_app_legacy:282-283)
                ko = os.path.join(out, "cuda_kernels_cu.o")
                _run([NVCC, *REF_NVCCFLAGS, "-I" + rinc, "-I" + srcdir, "-c", "-o", ko,
                      os.path.join(srcdir, "cuda", "cuda_kernels.cu")])
                pre_objs.append(ko)
                flags += ["-I" + os.path.join(CUDA_HOME, "include")]
        if name == "clover_step":
            objs_src.append(CLOVER_STEP_SRC)
        objs = []
        for p in objs_src:
            o = os.path.join(out, os.path.basename(p) + ".o")
            cmd = ["g++", *flags]
            if name == "clover_step" and os.path.basename(p).startswith("clover_leaf"):
                cmd += extra_defs
            if name == "clover_step" and p == CLOVER_STEP_SRC:
                cmd += ["-DCLOVER_STEP_REFERENCE"]
                if flavour == "ref_cuda":
                    cmd += ["-DCLOVER_STEP_CUDA", "-I" + os.path.join(CUDA_HOME, "include")]
            _run(cmd + ["-c", p, "-o", o])
            objs.append(o)
        link = ["g++", "-fopenmp", "-o", target, *pre_objs, *objs, lib]
        if flavour == "ref_cuda":
            # libops_cuda reads GPU power counters through NVML
            # (makefiles/Makefile.cuda:5): the driver's libnvidia-ml at run time
            link += ["-L" + os.path.join(CUDA_HOME, "lib64"), "-lcudart", "-lcurand",
                     "-L" + os.path.join(CUDA_HOME, "lib64", "stubs"), "-lnvidia-ml",
                     "-Wl,-rpath," + os.path.join(CUDA_HOME, "lib64")]
        if shared:
            link[1:1] = ["-shared", "-Wl,-Bsymbolic"]
        _run(link)
        return target
    raise ValueError(flavour)


def _build_b200_clover_step(out, d, paths, shared):
    from ops_b200.build_app import build as b200_build
    return b200_build("clover_step", out, paths, [d, APPS_DIR], defines=[], shared=shared,
                      rename_main={"clover_leaf.cpp": "clover_leaf_main"})


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("name")
    ap.add_argument("flavour")
    ap.add_argument("--shared", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.name, a.flavour, a.shared, a.force))


if __name__ == "__main__":
    main()
