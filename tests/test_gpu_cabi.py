"""The halo-transfer and batched-tridiagonal kernels driven through the C ABI
from this Python process (libops_b200.so loaded here), checked against numpy
restatements of the reference semantics.

Halo transfers must be bit-exact (copies); tridiagonal solves within 1e-12
relative (FP64) of an FP64 Thomas solve; FP32 storage within 2 float ulps.
"""

import ctypes as C

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def np_halo(src, dst, s_meta, d_meta, iters, fbase, tbase, fdir, tdir):
    """numpy model of one halo (ops_host_singlenode.cpp:172-446 semantics) on
    full arrays indexed [z][y][x] / [y][x]; meta = (d_m list)."""
    nd = len(iters)
    out = dst.copy()
    it = np.indices(iters[::-1]).reshape(nd, -1)[::-1]  # it[a] = coordinate along axis a
    def index(base, dirs, dm):
        idx = []
        for i in range(nd):
            ax = abs(dirs[i]) - 1
            t = it[ax] if dirs[i] > 0 else iters[ax] - 1 - it[ax]
            idx.append(base[i] - dm[i] + t)
        return tuple(idx[::-1])
    out[index(tbase, tdir, d_meta)] = src[index(fbase, fdir, s_meta)].astype(dst.dtype)
    return out


CASES_2D = [
    # iter, from_base, to_base, from_dir, to_dir
    ([1, 14], [11, 0], [-1, 0], [1, 2], [1, 2]),       # x face, same orientation
    ([12, 2], [0, 0], [0, 14], [1, 2], [1, 2]),        # 2-deep y face
    ([1, 15], [0, 0], [20, 0], [1, 2], [1, -2]),       # flipped along y
    ([10, 1], [2, 3], [-1, 0], [1, 2], [2, 1]),        # x of source -> y of target
    ([6, 4], [1, 2], [-2, -2], [-1, 2], [2, -1]),      # permuted and flipped, into halo corner
]


@pytest.mark.parametrize("case", range(len(CASES_2D)))
@pytest.mark.parametrize("types", [("double", "double"), ("float", "float"), ("double", "float")])
def test_halo_transfer_2d(case, types):
    from tests import cabi
    L = cabi.lib()
    b0 = L.ops_decl_block(2, b"hb0")
    b1 = L.ops_decl_block(2, b"hb1")
    src = cabi.Dat(b0, 2, [12, 20], [-2, -2], [2, 2], types[0], "src")
    dst = cabi.Dat(b1, 2, [20, 14], [-2, -2], [2, 2], types[1], "dst")
    rng = np.random.default_rng(case)
    s = rng.standard_normal(src.full_shape()).astype(src.dtype)
    d = rng.standard_normal(dst.full_shape()).astype(dst.dtype)
    src.set_full(s)
    dst.set_full(d)
    iters, fb, tb, fd, td = CASES_2D[case]
    h = L.ops_decl_halo(src.h, dst.h, cabi.ivec(iters), cabi.ivec(fb), cabi.ivec(tb),
                        cabi.ivec(fd), cabi.ivec(td))
    grp = L.ops_decl_halo_group(1, (C.c_void_p * 1)(h))
    L.ops_halo_transfer(grp)
    got = dst.get_full()
    want = np_halo(s, d, src.d_m, dst.d_m, iters, fb, tb, fd, td)
    assert np.array_equal(got, want)


def test_halo_group_3d_many():
    from tests import cabi
    L = cabi.lib()
    b = L.ops_decl_block(3, b"h3")
    a = cabi.Dat(b, 3, [9, 7, 5], [-1, -1, -1], [1, 1, 1], "double", "a3")
    c = cabi.Dat(b, 3, [7, 9, 6], [-1, -1, -1], [1, 1, 1], "double", "c3")
    rng = np.random.default_rng(7)
    sa, sc = rng.standard_normal(a.full_shape()), rng.standard_normal(c.full_shape())
    a.set_full(sa)
    c.set_full(sc)
    specs = [([1, 7, 5], [8, 0, 0], [-1, 0, 0], [1, 2, 3], [1, 2, 3]),
             ([7, 1, 5], [0, 0, 0], [0, 9, 0], [2, 1, 3], [1, 2, -3]),
             ([9, 7, 1], [0, 0, 4], [0, 0, -1], [1, 2, 3], [2, 1, 3])]
    hs = []
    want = sc
    for it, fb, tb, fd, td in specs:
        hs.append(L.ops_decl_halo(a.h, c.h, cabi.ivec(it), cabi.ivec(fb), cabi.ivec(tb),
                                  cabi.ivec(fd), cabi.ivec(td)))
        want = np_halo(sa, want, a.d_m, c.d_m, it, fb, tb, fd, td)
    grp = L.ops_decl_halo_group(len(hs), (C.c_void_p * len(hs))(*hs))
    L.ops_halo_transfer(grp)
    assert np.array_equal(c.get_full(), want)


def thomas(a, b, c, d):
    n = len(d)
    cp, dp = np.zeros(n), np.zeros(n)
    m = 1.0 / b[0]  # the oracle's order (oracle/src/oracle_trid.cpp)
    cp[0], dp[0] = c[0] * m, d[0] * m
    for i in range(1, n):
        m = 1.0 / (b[i] - a[i] * cp[i - 1])
        cp[i], dp[i] = c[i] * m, (d[i] - a[i] * dp[i - 1]) * m
    for i in range(n - 2, -1, -1):
        dp[i] -= cp[i] * dp[i + 1]
    return dp


def np_trid(A, B, Cc, D, U, solvedim, rng_box):
    """solve along axis solvedim (0=x) of [z][y][x] arrays inside the box"""
    X = D.copy() if U is None else U.copy()
    axis = 2 - solvedim
    sl = tuple(slice(rng_box[2 * (2 - k)], rng_box[2 * (2 - k) + 1]) for k in range(3))
    a, b, c, d = (np.moveaxis(M[sl].astype(np.float64), axis, -1) for M in (A, B, Cc, D))
    sol = np.empty_like(d)
    for idx in np.ndindex(d.shape[:-1]):
        sol[idx] = thomas(a[idx], b[idx], c[idx], d[idx])
    sol = np.moveaxis(sol, -1, axis)
    if U is None:
        X[sl] = sol.astype(X.dtype)
    else:
        X[sl] = (X[sl].astype(np.float64) + sol).astype(X.dtype)
    return X


@pytest.mark.parametrize("typ", ["double", "float"])
@pytest.mark.parametrize("solvedim", [0, 1, 2])
@pytest.mark.parametrize("inc", [False, True])
@pytest.mark.parametrize("shape", [(33, 7, 5), (7, 40, 3), (5, 6, 300), (2, 4, 3)])
def test_trid_batch(typ, solvedim, inc, shape, exact=False):
    from tests import cabi
    L = cabi.lib()
    blk = L.ops_decl_block(3, b"trid")
    nx, ny, nz = shape
    dats = {k: cabi.Dat(blk, 3, [nx, ny, nz], [-1, -1, -1], [1, 1, 1], typ, k)
            for k in "abcdu"}
    rng = np.random.default_rng(hash((typ, solvedim, inc, shape)) & 0xffff)
    full = dats["a"].full_shape()
    vals = {"a": rng.uniform(-1, 1, full), "c": rng.uniform(-1, 1, full),
            "b": 3.0 + rng.uniform(0, 1, full), "d": rng.uniform(-1, 1, full),
            "u": rng.uniform(-1, 1, full)}
    for k in "abcdu":
        vals[k] = vals[k].astype(dats[k].dtype)
        dats[k].set_full(vals[k])
    box = [0, nx, 0, ny, 0, nz]
    if nx > 3 and ny > 3:
        box = [1, nx - 1, 2, ny, 0, nz]  # a sub-range
    r = cabi.ivec(box)
    if inc:
        L.ops_tridMultiDimBatch_Inc(3, solvedim, r, dats["a"].h, dats["b"].h, dats["c"].h,
                                    dats["d"].h, dats["u"].h, None)
        got, target = dats["u"].get_full(), "u"
    else:
        L.ops_tridMultiDimBatch(3, solvedim, r, dats["a"].h, dats["b"].h, dats["c"].h,
                                dats["d"].h, None)
        got, target = dats["d"].get_full(), "d"
    # the storage box of the range: halo offset 1 in every axis
    sbox = [box[0] + 1, box[1] + 1, box[2] + 1, box[3] + 1, box[4] + 1, box[5] + 1]
    want = np_trid(vals["a"], vals["b"], vals["c"], vals["d"], vals["u"] if inc else None,
                   solvedim, sbox)
    if exact:
        assert np.array_equal(got, want)
    elif typ == "double":
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-13)
    else:
        np.testing.assert_allclose(got, want, rtol=2.5e-7, atol=1e-6)
    if inc:  # d untouched by the _Inc form
        assert np.array_equal(dats["d"].get_full(), vals["d"])


@pytest.mark.parametrize("typ", ["double", "float"])
@pytest.mark.parametrize("solvedim", [1, 2])
@pytest.mark.parametrize("inc", [False, True])
def test_trid_thomas_strided_bit_exact(typ, solvedim, inc):
    """OB2_TRID_STRIDED=0: strided lines solved one thread per line by the
    Thomas algorithm in the restatement's operation order without
    contraction: bit-identical to it (a child process, since the choice is
    read once per process)."""
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r); import tests.test_gpu_cabi as t; "
            "t.test_trid_batch(%r, %d, %r, (9, 37, 11), exact=True)" %
            (os.path.dirname(os.path.dirname(os.path.abspath(__file__))), typ, solvedim, inc))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       env=dict(os.environ, OB2_TRID_STRIDED="0"), timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]


@pytest.mark.parametrize("mode", ["1", "2", "3", "4"])
@pytest.mark.parametrize("typ", ["double", "float"])
def test_trid_strided_kernels(mode, typ):
    """Every kernel for strided lines -- OB2_TRID_STRIDED=1 the staged
    warp-per-line kernel, 2 and 3 the line-major CTA kernel with 16- and
    8-point chunks, 4 the line-major kernel with the warp PCR -- against the
    numpy Thomas model: y and z lines, with and
    without _Inc, line counts that do not fill the last CTA, line lengths
    from 5 to 200 (a child process per mode: the choice is read once)."""
    import subprocess
    import sys
    calls = "; ".join("t.test_trid_batch(%r, %d, %r, %r)" % (typ, sd, inc, shape)
                      for sd in (1, 2) for inc in (False, True)
                      for shape in ((9, 37, 11), (19, 5, 200), (33, 7, 5)))
    code = ("import sys; sys.path.insert(0, %r); import tests.test_gpu_cabi as t; %s" %
            (os.path.dirname(os.path.dirname(os.path.abspath(__file__))), calls))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       env=dict(os.environ, OB2_TRID_STRIDED=mode), timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]


def test_device_memspace_slab_set_and_fetch():
    """The external data access API with device buffers (OPS_DEVICE), as the
    reference's access app uses it (apps/c/access/fetch_data.cu): a 2 x 2 slab
    set from device memory, the whole interior and another slab fetched into
    device memory, checked against numpy."""
    from tests import cabi
    L = cabi.lib()
    vp, ip = C.c_void_p, C.POINTER(C.c_int)
    L.ops_dat_set_data_slab_memspace.argtypes = [vp, C.c_int, vp, ip, C.c_int]
    L.ops_dat_fetch_data_slab_memspace.argtypes = [vp, C.c_int, vp, ip, C.c_int]
    L.ops_dat_fetch_data_memspace.argtypes = [vp, C.c_int, vp, C.c_int]
    L.ob2_dev_malloc.argtypes = [C.POINTER(vp), C.c_size_t]
    L.ob2_dev_free.argtypes = [vp]
    L.ob2_dev_h2d.argtypes = [vp, vp, C.c_size_t]
    L.ob2_dev_d2h.argtypes = [vp, vp, C.c_size_t]
    OPS_DEVICE = 2
    blk = L.ops_decl_block(2, b"access")
    dat = cabi.Dat(blk, 2, [20, 20], [-1, -1], [1, 1], "double", "data0")
    interior = np.add.outer(100.0 * np.arange(20), np.arange(20.0))  # [y, x] = x + 100 y
    dat.set_interior(interior)
    want = interior.copy()

    def dev(nbytes):
        p = vp()
        assert L.ob2_dev_malloc(C.byref(p), nbytes) == 0
        return p

    slab_in = np.array([-1.0, -2.0, -3.0, -4.0])
    d_in = dev(32)
    assert L.ob2_dev_h2d(d_in, slab_in.ctypes.data, 32) == 0
    L.ops_dat_set_data_slab_memspace(dat.h, 0, d_in, cabi.ivec([6, 8, 6, 8]), OPS_DEVICE)
    want[6:8, 6:8] = slab_in.reshape(2, 2)

    d_all = dev(20 * 20 * 8)
    L.ops_dat_fetch_data_memspace(dat.h, 0, d_all, OPS_DEVICE)
    got = np.empty((20, 20))
    assert L.ob2_dev_d2h(got.ctypes.data, d_all, got.nbytes) == 0
    assert np.array_equal(got, want)

    d_slab = dev(32)
    L.ops_dat_fetch_data_slab_memspace(dat.h, 0, d_slab, cabi.ivec([10, 12, 10, 12]), OPS_DEVICE)
    slab_out = np.empty(4)
    assert L.ob2_dev_d2h(slab_out.ctypes.data, d_slab, 32) == 0
    assert np.array_equal(slab_out, want[10:12, 10:12].ravel())
    for p in (d_in, d_all, d_slab):
        L.ob2_dev_free(p)


@pytest.mark.parametrize("mode", ["0", "1"])
@pytest.mark.parametrize("typ", ["double", "float"])
def test_trid_unit_stride_kernels(mode, typ):
    """Unit-stride (x) lines: OB2_TRID_UNIT=1 the vectorised warp-per-line
    kernel (16-, 8- or 4-byte accesses as each line's alignment allows, the
    partial last chunk element by element), 0 the scalar one, against the
    numpy Thomas model: line lengths 2 to 256 (odd lengths, the halo making
    every line start off 16-byte alignment), with and without _Inc, line
    counts that do not fill the last CTA (a child process per mode)."""
    import subprocess
    import sys
    calls = "; ".join("t.test_trid_batch(%r, 0, %r, %r)" % (typ, inc, shape)
                      for inc in (False, True)
                      for shape in ((256, 3, 5), (255, 4, 3), (64, 9, 2), (2, 5, 7), (131, 2, 2),
                                   (300, 2, 2)))
    code = ("import sys; sys.path.insert(0, %r); import tests.test_gpu_cabi as t; %s" %
            (os.path.dirname(os.path.dirname(os.path.abspath(__file__))), calls))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       env=dict(os.environ, OB2_TRID_UNIT=mode), timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
