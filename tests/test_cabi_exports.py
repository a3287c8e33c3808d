"""The C-ABI library loads (no GPU needed) and exports every entry point the
public headers declare."""

import ctypes
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "ops_b200", "lib", "libops_b200.so")


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "ops_b200"), "-j8"], check=True)
    return LIB


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = "\n".join(l for l in text.splitlines() if not l.lstrip().startswith("#"))
        for m in re.finditer(r"\b(?:OPS_API|OB2_API)\s+[\w\s\*]+?\b(\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_headers_declare_the_api():
    names = declared_symbols()
    for must in ("ops_init", "ops_decl_dat_char", "ops_arg_dat", "ops_halo_transfer",
                 "ops_reduction_result_char", "ops_tridMultiDimBatch", "ops_tridMultiDimBatch_Inc",
                 "ob2_loop_begin", "ob2_trid_batch", "ob2_halo_run"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True,
                         check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if l.strip()}
    missing = sorted(declared_symbols() - exported)
    assert not missing, missing


def test_library_loads_without_gpu(lib):
    L = ctypes.CDLL(lib)
    # resolving symbols performs no CUDA work
    for name in ("ops_init", "ob2_loop_begin", "ops_dat_fetch_data", "ob2_halo_run_noalloc"):
        assert hasattr(L, name)
