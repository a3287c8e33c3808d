"""ctypes view of the C ABI of libops_b200.so (include/ops_lib_core.h,
include/ops_tridiag.h), for tests that drive the runtime directly from
Python: declare blocks and dats, move data, run halo transfers and batched
tridiagonal solves, read dats back with halos."""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "ops_b200", "lib", "libops_b200.so")

_L = None
_NP = {"double": (np.float64, 8), "float": (np.float32, 4), "int": (np.int32, 4)}


def lib():
    global _L
    if _L is None:
        L = C.CDLL(LIB, mode=C.RTLD_GLOBAL)
        vp, ip = C.c_void_p, C.POINTER(C.c_int)
        L.ops_init.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.c_int]
        L.ops_decl_block.restype = vp
        L.ops_decl_block.argtypes = [C.c_int, C.c_char_p]
        L.ops_decl_dat_char.restype = vp
        L.ops_decl_dat_char.argtypes = [vp, C.c_int, ip, ip, ip, ip, ip, C.c_char_p, C.c_int,
                                        C.c_char_p, C.c_char_p]
        L.ops_decl_halo.restype = vp
        L.ops_decl_halo.argtypes = [vp, vp, ip, ip, ip, ip, ip]
        L.ops_decl_halo_group.restype = vp
        L.ops_decl_halo_group.argtypes = [C.c_int, C.POINTER(vp)]
        L.ops_halo_transfer.argtypes = [vp]
        L.ops_dat_get_raw_pointer.restype = C.c_void_p
        L.ops_dat_get_raw_pointer.argtypes = [vp, C.c_int, vp, ip]
        L.ops_dat_release_raw_data.argtypes = [vp, C.c_int, C.c_int]
        L.ops_dat_get_raw_metadata.argtypes = [vp, C.c_int, ip, ip, ip, ip, ip]
        L.ops_dat_set_data.argtypes = [vp, C.c_int, vp]
        L.ops_dat_fetch_data.argtypes = [vp, C.c_int, vp]
        L.ops_tridMultiDimBatch.argtypes = [C.c_int, C.c_int, ip, vp, vp, vp, vp, vp]
        L.ops_tridMultiDimBatch_Inc.argtypes = [C.c_int, C.c_int, ip, vp, vp, vp, vp, vp, vp]
        argv = (C.c_char_p * 2)(b"cabi", None)
        L.ops_init(1, argv, 1)
        _L = L
    return _L


def ivec(vals):
    return (C.c_int * len(vals))(*vals)


class Dat:
    """An ops_dat declared through ops_decl_dat_char (OPS-allocated)."""

    def __init__(self, block, ndim, size, d_m, d_p, typ="double", name="d"):
        L = lib()
        self.ndim, self.size, self.d_m, self.d_p, self.typ = ndim, list(size), list(d_m), list(d_p), typ
        dt, ts = _NP[typ]
        self.dtype = dt
        self.h = L.ops_decl_dat_char(block, 1, ivec(size), ivec([0] * ndim), ivec(d_m), ivec(d_p),
                                     ivec([1] * ndim), None, ts, typ.encode(), name.encode())

    def full_shape(self):
        # numpy shape (slowest first) of the allocation, halos included
        return tuple(s - m + p for s, m, p in zip(self.size, self.d_m, self.d_p))[::-1]

    def set_interior(self, arr):
        a = np.ascontiguousarray(arr, dtype=self.dtype)
        assert a.shape == tuple(self.size[::-1])
        lib().ops_dat_set_data(self.h, 0, a.ctypes.data)

    def set_full(self, arr):
        """Whole allocation (halos included) through the host raw pointer."""
        a = np.ascontiguousarray(arr, dtype=self.dtype)
        view = self._raw(C.c_int(1))
        view[...] = a
        lib().ops_dat_release_raw_data(self.h, 0, 2)  # OPS_RW: host copy is newer

    def get_full(self):
        view = self._raw(C.c_int(1))
        out = view.copy()
        lib().ops_dat_release_raw_data(self.h, 0, 0)  # OPS_READ
        return out

    def _raw(self, ms):
        L = lib()
        p = L.ops_dat_get_raw_pointer(self.h, 0, None, C.byref(ms))
        stride = (C.c_int * 3)()
        dm = (C.c_int * 3)()
        L.ops_dat_get_raw_metadata(self.h, 0, None, None, stride, dm, None)
        strides = [stride[i] for i in range(self.ndim)]
        off = 0
        cum = 1
        for i in range(self.ndim):
            off += dm[i] * cum
            cum *= strides[i]
        itemsize = np.dtype(self.dtype).itemsize
        base = p + off * itemsize
        n = int(np.prod(strides))
        buf = (C.c_char * (n * itemsize)).from_address(base)
        return np.frombuffer(buf, dtype=self.dtype).reshape(tuple(strides[::-1]))
