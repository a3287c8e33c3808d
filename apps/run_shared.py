"""Run an OPS application built as a shared library inside this Python process.

    python -m apps.run_shared NAME FLAVOUR [app args...]

The library (built with --shared, `main` renamed to `ops_app_main`) is loaded
with ctypes and its main is called, so the backend's shared library
(libops_b200.so for the b200 flavour) is loaded by this process.  One OPS
application per process: the OPS runtime state is process-global.
"""

from __future__ import annotations

import ctypes
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def app_entry(L):
    """The app's renamed main: `int ops_app_main(int, char **)` (C++ linkage,
    Itanium-mangled)."""
    for sym in ("ops_app_main", "_Z12ops_app_mainiPPc"):
        try:
            f = getattr(L, sym)
        except AttributeError:
            continue
        f.restype = ctypes.c_int
        return f
    raise AttributeError("no ops_app_main in the library")


def run(name: str, flavour: str, args) -> int:
    from apps.catalog import artifact, build
    lib = artifact(name, flavour, shared=True)
    if not os.path.exists(lib):
        lib = build(name, flavour, shared=True)
    L = ctypes.CDLL(lib, mode=ctypes.RTLD_GLOBAL)
    argv = [name.encode()] + [a.encode() for a in args]
    arr = (ctypes.c_char_p * (len(argv) + 1))(*argv, None)
    entry = app_entry(L)
    rc = entry(len(argv), arr)
    sys.stdout.flush()
    return rc


if __name__ == "__main__":
    if len(sys.argv) < 3:
        raise SystemExit(__doc__)
    sys.exit(run(sys.argv[1], sys.argv[2], sys.argv[3:]))
