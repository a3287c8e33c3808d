"""The division that translated user kernels use (ob2::ddiv,
include/ops_b200_kernel.h) against CUDA's IEEE `/`, bit for bit, on the GPU.

The harness (tests/gpu_src/ddiv_check.cu, built by __graft_entry__.build()
into tests/_build/) draws operand pairs from a counter-based hash: operands
anywhere in the fast domain, quotients next to rounding midpoints, zero
numerators of both signs, divisors whose significands are near all ones or
powers of two, and arbitrary bit patterns (the IEEE fallback)."""

import ctypes
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "tests", "_build", "libddiv_check.so")

pytestmark = pytest.mark.gpu

MODES = {0: "fast domain", 1: "near midpoints", 2: "zero numerators, integers",
         3: "divisors near all-ones significands", 4: "any bit pattern"}


@pytest.mark.parametrize("mode", sorted(MODES))
def test_ddiv_equals_ieee_division(mode):
    assert os.path.exists(LIB), "harness not built: " + LIB
    L = ctypes.CDLL(LIB)
    L.ddiv_check.argtypes = [ctypes.c_ulonglong, ctypes.c_ulonglong, ctypes.c_int,
                             ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(ctypes.c_double)]
    bad = ctypes.c_ulonglong(0)
    first = (ctypes.c_double * 3)()
    n = 1 << 30
    for seed in (1, 2):
        rc = L.ddiv_check(n, seed * 7919 + mode, mode, ctypes.byref(bad), first)
        assert rc == 0, "CUDA error %d" % rc
        assert bad.value == 0, "%s: %d of %d quotients differ, e.g. %r / %r -> %r" % (
            MODES[mode], bad.value, n, first[0], first[1], first[2])
