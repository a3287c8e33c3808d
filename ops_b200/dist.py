"""Host transport for the slab decomposition (include/ops_b200_dist.h) over a
torch.distributed process group (gloo: CPU tensors, any number of ranks on
one machine or several).

    import torch.distributed as dist
    dist.init_process_group("gloo")
    from ops_b200.dist import install
    install(ctypes.CDLL(".../libops_b200.so"))   # before ops_init

The runtime stages the rows it exchanges through pinned host memory and
calls back into this module; every rank takes the same calls in the same
order (the exchanges follow the program's loops, the reductions its
ops_reduction_result calls).
"""

from __future__ import annotations

import ctypes

SENDRECV = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                            ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int)
ALLREDUCE = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                             ctypes.c_int, ctypes.c_int)


class Comm(ctypes.Structure):
    """Mirror of ob2_dist_comm."""
    _fields_ = [("rank", ctypes.c_int), ("size", ctypes.c_int), ("device", ctypes.c_int),
                ("ctx", ctypes.c_void_p), ("sendrecv", SENDRECV), ("allreduce", ALLREDUCE)]


_keep = []  # the callbacks must outlive the library's use of them

OPS_INC, OPS_MIN, OPS_MAX = 3, 4, 5


def _tensor(ptr, nbytes):
    import torch
    buf = (ctypes.c_char * nbytes).from_address(ptr)
    return torch.frombuffer(buf, dtype=torch.uint8)


def _sendrecv(ctx, sbuf, sbytes, speer, rbuf, rbytes, rpeer):
    import torch.distributed as dist
    try:
        reqs = []
        if sbytes and speer >= 0:
            reqs.append(dist.isend(_tensor(sbuf, sbytes), dst=speer))
        if rbytes and rpeer >= 0:
            reqs.append(dist.irecv(_tensor(rbuf, rbytes), src=rpeer))
        for r in reqs:
            r.wait()
        return 0
    except Exception:  # noqa: BLE001 - the runtime turns a non-zero into an OPSException
        return 1


def _allreduce(ctx, buf, count, typ, op):
    import torch
    import torch.distributed as dist
    try:
        dt, size = {0: (torch.float64, 8), 1: (torch.float32, 4), 2: (torch.int32, 4),
                    3: (torch.int64, 8)}[typ]
        t = _tensor(buf, count * size).view(dt)
        rop = {OPS_INC: dist.ReduceOp.SUM, OPS_MIN: dist.ReduceOp.MIN,
               OPS_MAX: dist.ReduceOp.MAX}[op]
        dist.all_reduce(t, op=rop)
        return 0
    except Exception:  # noqa: BLE001
        return 1


def install(lib) -> int:
    """Registers the current process group as lib's communicator (lib:
    libops_b200.so or any library exporting ob2_dist_init)."""
    import torch.distributed as dist
    c = Comm()
    c.rank = dist.get_rank()
    c.size = dist.get_world_size()
    c.device = 0
    c.ctx = None
    c.sendrecv = SENDRECV(_sendrecv)
    c.allreduce = ALLREDUCE(_allreduce)
    _keep.append(c)
    lib.ob2_dist_init.argtypes = [ctypes.POINTER(Comm)]
    return lib.ob2_dist_init(ctypes.byref(c))
