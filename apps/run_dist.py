"""Run an OPS application built as a shared library on several ranks with
the slab decomposition (include/ops_b200_dist.h) and a gloo host transport.

    RANK=r WORLD_SIZE=n MASTER_ADDR=127.0.0.1 MASTER_PORT=p \\
        python -m apps.run_dist NAME FLAVOUR [app args...]

(or under torchrun).  The process group is gloo on CPU tensors; the
backend library of the flavour (libops_b200.so or the oracle's) gets the
communicator before the application's ops_init.  OPS_DUMP_FILE, when set,
receives one dump per rank (suffix .r<rank>) of the rows that rank owns.
"""

from __future__ import annotations

import ctypes
import datetime
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main(argv) -> int:
    import torch.distributed as dist

    from apps.catalog import ORACLE_LIB_DIR, artifact, build
    from apps.run_shared import app_entry
    from ops_b200.dist import install
    name, flavour, args = argv[0], argv[1], argv[2:]
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    try:
        lib = artifact(name, flavour, shared=True)
        if not os.path.exists(lib):
            lib = build(name, flavour, shared=True)
        backend = (os.path.join(ROOT, "ops_b200", "lib", "libops_b200.so") if flavour == "b200"
                   else os.path.join(ORACLE_LIB_DIR, "liboracle_ops.so"))
        B = ctypes.CDLL(backend, mode=ctypes.RTLD_GLOBAL)
        if install(B) != 0:
            raise RuntimeError("ob2_dist_init refused the communicator")
        L = ctypes.CDLL(lib, mode=ctypes.RTLD_GLOBAL)
        av = [name.encode()] + [a.encode() for a in args]
        arr = (ctypes.c_char_p * (len(av) + 1))(*av, None)
        rc = app_entry(L)(len(av), arr)
        sys.stdout.flush()
        dist.barrier()
        return rc
    finally:
        dist.destroy_process_group()


if __name__ == "__main__":
    if len(sys.argv) < 3:
        raise SystemExit(__doc__)
    sys.exit(main(sys.argv[1:]))
