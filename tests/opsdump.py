"""Reader and comparator for the dat dump files written at ops_exit when
OPS_DUMP_FILE is set (same binary format from the B200 runtime and from the
CPU oracle): every live dat, halos included."""

from __future__ import annotations

import struct
from typing import Dict, Tuple

import numpy as np

_NP = {"double": np.float64, "float": np.float32, "int": np.int32, "long long": np.int64,
       "ll": np.int64, "half": np.float16}


def read_dump(path: str, mmap: bool = False) -> Dict[str, Tuple[dict, np.ndarray]]:
    """Every record of a dump file; mmap=True maps the data instead of reading
    it (dumps of full-size configurations are gigabytes)."""
    out = {}
    with open(path, "rb") as f:
        data = f.read() if not mmap else None
    if mmap:
        import mmap as _mm
        fh = open(path, "rb")
        data = _mm.mmap(fh.fileno(), 0, access=_mm.ACCESS_READ)
    o = 0
    while o < len(data):
        assert data[o:o + 4] == b"DAT0", "bad dump record at %d" % o
        o += 4
        (nl,) = struct.unpack_from("i", data, o); o += 4
        name = data[o:o + nl].decode(); o += nl
        (tl,) = struct.unpack_from("i", data, o); o += 4
        typ = data[o:o + tl].decode(); o += tl
        dim, ts, ndims, soa = struct.unpack_from("4i", data, o); o += 16
        size = struct.unpack_from("5i", data, o); o += 20
        d_m = struct.unpack_from("5i", data, o); o += 20
        d_p = struct.unpack_from("5i", data, o); o += 20
        (nb,) = struct.unpack_from("Q", data, o); o += 8
        dt = _NP.get(typ)
        if mmap:
            arr = np.memmap(path, dtype=dt if dt is not None else np.uint8, mode="r", offset=o,
                            shape=(nb // (np.dtype(dt).itemsize if dt is not None else 1),))
        else:
            raw = data[o:o + nb]
            arr = (np.frombuffer(raw, dtype=dt) if dt is not None
                   else np.frombuffer(raw, np.uint8)).copy()
        o += nb
        meta = {"type": typ, "dim": dim, "ndims": ndims, "size": size[:ndims], "d_m": d_m[:ndims],
                "d_p": d_p[:ndims], "soa": soa}
        key = name
        k = 1
        while key in out:
            key = "%s#%d" % (name, k)
            k += 1
        out[key] = (meta, arr)
    return out


def compare(a_path: str, b_path: str, rtol: float = 1e-12, exact_types=("int",),
            skip=(), floor_frac: float = 1e-3, mmap: bool = False,
            chunk: int = 1 << 24) -> Dict[str, float]:
    """Max relative difference per dat, |a-b| / max(|b|, floor_frac * max|b|);
    floor_frac = 1 gives the error relative to the field's scale.  Raises on
    shape/type mismatch; integer dats must match exactly.  mmap=True maps
    both files and works through each dat in chunks of `chunk` elements."""
    A, Bd = read_dump(a_path, mmap), read_dump(b_path, mmap)
    assert set(A) == set(Bd), "dat sets differ: %s" % (set(A) ^ set(Bd))
    res = {}
    for name in A:
        if any(s in name for s in skip):
            continue
        ma, xa = A[name]
        mb, xb = Bd[name]
        assert ma["size"] == mb["size"] and ma["type"] == mb["type"], name
        assert xa.size == xb.size, name
        if ma["type"] in exact_types:
            same = all(np.array_equal(xa[i:i + chunk], xb[i:i + chunk])
                       for i in range(0, xa.size, chunk))
            res[name] = 0.0 if same else float("inf")
            continue
        scale = 0.0
        for i in range(0, xb.size, chunk):
            scale = max(scale, float(np.max(np.abs(xb[i:i + chunk].astype(np.float64)))))
        scale = max(scale, 1e-300)
        worst = 0.0
        for i in range(0, xa.size, chunk):
            a = xa[i:i + chunk].astype(np.float64)
            b = xb[i:i + chunk].astype(np.float64)
            # per element relative with an absolute floor relative to the field scale
            rel = np.abs(a - b) / np.maximum(np.abs(b), floor_frac * scale)
            if rel.size:
                worst = max(worst, float(np.max(rel)))
        res[name] = worst
    return res
