"""Reader and comparator for the dat dump files written at ops_exit when
OPS_DUMP_FILE is set (same binary format from the B200 runtime and from the
CPU oracle): every live dat, halos included."""

from __future__ import annotations

import struct
from typing import Dict, Tuple

import numpy as np

_NP = {"double": np.float64, "float": np.float32, "int": np.int32, "long long": np.int64,
       "ll": np.int64}


def read_dump(path: str) -> Dict[str, Tuple[dict, np.ndarray]]:
    out = {}
    with open(path, "rb") as f:
        data = f.read()
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
        raw = data[o:o + nb]; o += nb
        dt = _NP.get(typ)
        arr = np.frombuffer(raw, dtype=dt) if dt is not None else np.frombuffer(raw, np.uint8)
        meta = {"type": typ, "dim": dim, "ndims": ndims, "size": size[:ndims], "d_m": d_m[:ndims],
                "d_p": d_p[:ndims], "soa": soa}
        key = name
        k = 1
        while key in out:
            key = "%s#%d" % (name, k)
            k += 1
        out[key] = (meta, arr.copy())
    return out


def compare(a_path: str, b_path: str, rtol: float = 1e-12, exact_types=("int",),
            skip=(), floor_frac: float = 1e-3) -> Dict[str, float]:
    """Max relative difference per dat, |a-b| / max(|b|, floor_frac * max|b|);
    floor_frac = 1 gives the error relative to the field's scale.  Raises on
    shape/type mismatch; integer dats must match exactly."""
    A, Bd = read_dump(a_path), read_dump(b_path)
    assert set(A) == set(Bd), "dat sets differ: %s" % (set(A) ^ set(Bd))
    res = {}
    for name in A:
        if any(s in name for s in skip):
            continue
        ma, xa = A[name]
        mb, xb = Bd[name]
        assert ma["size"] == mb["size"] and ma["type"] == mb["type"], name
        if ma["type"] in exact_types:
            res[name] = 0.0 if np.array_equal(xa, xb) else float("inf")
            continue
        xa = xa.astype(np.float64)
        xb = xb.astype(np.float64)
        scale = max(float(np.max(np.abs(xb))) if xb.size else 0.0, 1e-300)
        diff = np.abs(xa - xb)
        # per element relative with an absolute floor relative to the field scale
        rel = diff / np.maximum(np.abs(xb), floor_frac * scale)
        res[name] = float(np.max(rel)) if rel.size else 0.0
    return res
