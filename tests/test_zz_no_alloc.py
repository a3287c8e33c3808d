"""ob2_halo_run_noalloc: the halo transfer for callers that cannot allocate
device memory (their memory budget belongs to someone else, or they run where
allocations are not allowed).  Its task table sits in a fixed array inside
libops_b200.so instead of memory the caller allocates.

Checked through the C ABI against ob2_halo_run (caller-allocated table) and
against the numpy model of the reference's halo semantics on the same inputs,
on two calls in a row with different tables, with a table of exactly the
maximum size, and against its error returns (a table above the maximum, a
negative count).  Halo copies are exact, so the outputs must be identical.
This file is collected last and also runs alone in a fresh process.
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


class HaloTask(C.Structure):
    """Mirror of ob2_halo_task (include/ops_b200_device.h)."""
    _fields_ = [("src", C.c_void_p), ("dst", C.c_void_p), ("src_type", C.c_int),
                ("dst_type", C.c_int), ("ncomp", C.c_int), ("src_soa", C.c_int),
                ("dst_soa", C.c_int), ("iter", C.c_int * 3), ("npts", C.c_longlong),
                ("src_axis", C.c_int * 3), ("src_flip", C.c_int * 3), ("src_start", C.c_int * 3),
                ("src_cum", C.c_longlong * 3), ("dst_axis", C.c_int * 3),
                ("dst_flip", C.c_int * 3), ("dst_start", C.c_int * 3),
                ("dst_cum", C.c_longlong * 3), ("src_npts_total", C.c_longlong),
                ("dst_npts_total", C.c_longlong), ("float_kind", C.c_int)]


OB2_HALO_STATIC_MAX = 1024
OB2_ERR_NOALLOC_LIMIT = 100001


def device_base(dat):
    """Device address of the dat's allocation (halos included); leaves the
    runtime believing the device copy is the newer one."""
    from tests import cabi
    L = cabi.lib()
    ms = C.c_int(2)  # OPS_DEVICE: uploads the host copy written by set_full
    p = L.ops_dat_get_raw_pointer(dat.h, 0, None, C.byref(ms))
    L.ops_dat_release_raw_data_memspace.argtypes = [C.c_void_p, C.c_int, C.c_int,
                                                    C.POINTER(C.c_int)]
    L.ops_dat_release_raw_data_memspace(dat.h, 0, 2, C.byref(ms))  # OPS_RW on the device
    off, cum = 0, 1
    full = dat.full_shape()[::-1]
    for i in range(dat.ndim):
        off += -dat.d_m[i] * cum
        cum *= full[i]
    return p - off * np.dtype(dat.dtype).itemsize


def make_task(src, dst, sbase, dbase, iters, fb, tb, fd, td):
    t = HaloTask()
    t.src, t.dst = sbase, dbase
    t.src_type = t.dst_type = np.dtype(src.dtype).itemsize
    t.ncomp = 1
    t.npts = int(np.prod(iters))
    sfull, dfull = src.full_shape()[::-1], dst.full_shape()[::-1]
    sc = dc = 1
    for i in range(3):
        t.iter[i] = iters[i] if i < len(iters) else 1
    for i in range(3):
        used = i < src.ndim
        t.src_axis[i] = abs(fd[i]) - 1 if used else i
        t.src_flip[i] = int(used and fd[i] < 0)
        t.src_start[i] = (fb[i] - src.d_m[i]) if used else 0
        t.src_cum[i] = sc
        sc *= sfull[i] if used else 1
        t.dst_axis[i] = abs(td[i]) - 1 if used else i
        t.dst_flip[i] = int(used and td[i] < 0)
        t.dst_start[i] = (tb[i] - dst.d_m[i]) if used else 0
        t.dst_cum[i] = dc
        dc *= dfull[i] if used else 1
    t.src_npts_total, t.dst_npts_total = sc, dc
    return t


def run_both(tasks, src, dst, s0, d0):
    """Run the tasks with ob2_halo_run and with ob2_halo_run_noalloc from the
    same starting data; return both results."""
    from tests import cabi
    L = cabi.lib()
    L.ob2_halo_run.argtypes = [C.c_void_p, C.c_int, C.c_longlong]
    L.ob2_halo_run_noalloc.argtypes = [C.c_void_p, C.c_int]
    L.ob2_dev_malloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
    L.ob2_dev_h2d.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
    L.ob2_dev_free.argtypes = [C.c_void_p]
    arr = (HaloTask * len(tasks))(*tasks)
    nbytes = C.sizeof(arr)
    max_pts = max(t.npts for t in tasks)

    src.set_full(s0)
    dst.set_full(d0)
    sb, db = device_base(src), device_base(dst)
    for t in arr:
        t.src, t.dst = sb, db
    table = C.c_void_p()
    assert L.ob2_dev_malloc(C.byref(table), nbytes) == 0
    assert L.ob2_dev_h2d(table, arr, nbytes) == 0
    assert L.ob2_halo_run(table, len(tasks), max_pts) == 0
    assert L.ob2_dev_sync() == 0
    with_alloc = dst.get_full()
    L.ob2_dev_free(table)

    dst.set_full(d0)
    sb, db = device_base(src), device_base(dst)
    for t in arr:
        t.src, t.dst = sb, db
    assert L.ob2_halo_run_noalloc(arr, len(tasks)) == 0
    assert L.ob2_dev_sync() == 0
    return with_alloc, dst.get_full()


def model(tasks_spec, src, dst, s0, d0):
    """The numpy model of the reference's halo semantics applied task by task
    (tests/test_gpu_cabi.py: np_halo)."""
    from tests.test_gpu_cabi import np_halo
    out = d0.copy()
    for iters, fb, tb, fd, td in tasks_spec:
        out = np_halo(s0, out, src.d_m, dst.d_m, iters, fb, tb, fd, td)
    return out


def test_noalloc_matches_allocating_entry_twice():
    from tests import cabi
    L = cabi.lib()
    b = L.ops_decl_block(2, b"noalloc")
    src = cabi.Dat(b, 2, [24, 18], [-2, -2], [2, 2], "double", "na_src")
    dst = cabi.Dat(b, 2, [18, 30], [-2, -2], [2, 2], "double", "na_dst")
    rng = np.random.default_rng(11)
    s0 = rng.standard_normal(src.full_shape())
    d0 = rng.standard_normal(dst.full_shape())
    spec1 = [([6, 4], [1, 2], [-2, -2], [-1, 2], [2, -1]),
             ([1, 18], [23, 0], [-1, 0], [1, 2], [2, 1])]
    first = [make_task(src, dst, 0, 0, *t) for t in spec1]
    a1, n1 = run_both(first, src, dst, s0, d0)
    assert np.array_equal(a1, n1)
    assert np.array_equal(n1, model(spec1, src, dst, s0, d0))
    assert not np.array_equal(a1, d0)  # the halos really moved data
    # a second call with a different (smaller) table: nothing of the first
    # call's table may leak into it
    spec2 = [([18, 2], [3, 0], [0, 30], [2, 1], [1, 2])]
    second = [make_task(src, dst, 0, 0, *t) for t in spec2]
    a2, n2 = run_both(second, src, dst, s0, d0)
    assert np.array_equal(a2, n2)
    assert np.array_equal(n2, model(spec2, src, dst, s0, d0))
    assert not np.array_equal(a2, a1)


def test_noalloc_full_table_of_the_maximum_size():
    """Exactly OB2_HALO_STATIC_MAX one-point tasks (the accepted upper edge):
    point k of a 32 x 32 block of the source goes to the transposed point of
    the target."""
    from tests import cabi
    L = cabi.lib()
    b = L.ops_decl_block(2, b"noalloc_max")
    src = cabi.Dat(b, 2, [32, 32], [0, 0], [0, 0], "double", "nm_src")
    dst = cabi.Dat(b, 2, [32, 32], [0, 0], [0, 0], "double", "nm_dst")
    rng = np.random.default_rng(5)
    s0 = rng.standard_normal(src.full_shape())
    d0 = rng.standard_normal(dst.full_shape())
    spec = [([1, 1], [k % 32, k // 32], [k // 32, k % 32], [1, 2], [1, 2])
            for k in range(OB2_HALO_STATIC_MAX)]
    tasks = [make_task(src, dst, 0, 0, *t) for t in spec]
    a, n = run_both(tasks, src, dst, s0, d0)
    assert np.array_equal(a, n)
    assert np.array_equal(n, s0.T)
    assert np.array_equal(n, model(spec, src, dst, s0, d0))


def test_noalloc_rejects_tables_above_the_limit():
    from tests import cabi
    L = cabi.lib()
    L.ob2_halo_run_noalloc.argtypes = [C.c_void_p, C.c_int]
    L.ob2_error_string.restype = C.c_char_p
    big = (HaloTask * (OB2_HALO_STATIC_MAX + 1))()
    rc = L.ob2_halo_run_noalloc(big, OB2_HALO_STATIC_MAX + 1)
    assert rc == OB2_ERR_NOALLOC_LIMIT
    assert b"maximum" in L.ob2_error_string(rc)
    assert L.ob2_dev_sync() == 0


def test_noalloc_rejects_a_negative_count_without_launching():
    from tests import cabi
    L = cabi.lib()
    L.ob2_halo_run_noalloc.argtypes = [C.c_void_p, C.c_int]
    L.ob2_error_string.restype = C.c_char_p
    b = L.ops_decl_block(2, b"noalloc_neg")
    src = cabi.Dat(b, 2, [8, 8], [0, 0], [0, 0], "double", "nn_src")
    dst = cabi.Dat(b, 2, [8, 8], [0, 0], [0, 0], "double", "nn_dst")
    d0 = np.arange(64, dtype=np.float64).reshape(8, 8)
    src.set_full(-d0)
    dst.set_full(d0)
    t = make_task(src, dst, device_base(src), device_base(dst), [8, 8], [0, 0], [0, 0],
                  [1, 2], [1, 2])
    one = (HaloTask * 1)(t)
    rc = L.ob2_halo_run_noalloc(one, -1)
    assert rc == 1  # cudaErrorInvalidValue
    assert b"maximum" not in L.ob2_error_string(rc)
    assert L.ob2_dev_sync() == 0
    assert np.array_equal(dst.get_full(), d0)  # nothing was copied
