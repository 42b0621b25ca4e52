"""One bunch split over several processes (one GPU each) by particle range.

The reference runs a bunch over MPI ranks: each rank tracks its own
particles and the ranks exchange the moment sums of the adaptive domain,
the valid counts of update_total_num and the charge density of every
deposit.  Here each rank owns a Propagator and a Bunch holding its shard;
`attach` gives the propagator a torch.distributed sum-allreduce for those
exchanges (sb2_propagator_set_allreduce).
"""
import numpy as np


def shard_range(n, rank, world):
    """Contiguous particle range [lo, hi) of `rank` among `world` ranks."""
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def attach(propagator, group=None, on_host=None):
    """Give `propagator` a torch.distributed sum-allreduce over `group`.
    on_host (default: True for the gloo backend, False for NCCL) selects host
    staging or device buffers.  The callback is typed, so a mixed-precision
    propagator sums its FP32 charge grid as float32."""
    import torch
    import torch.distributed as dist
    if on_host is None:
        on_host = dist.get_backend(group) != "nccl"
    if torch.cuda.is_available():  # the library's own (static) CUDA runtime follows torch's device
        from . import _lib
        _lib.check(_lib.lib().sb2_set_device(torch.cuda.current_device()))
    if on_host:
        def fn(arr):
            dist.all_reduce(torch.from_numpy(arr), op=dist.ReduceOp.SUM, group=group)
    else:
        class _Dev:  # a device buffer seen through __cuda_array_interface__
            def __init__(self, ptr, n, dtype):
                self.__cuda_array_interface__ = {"shape": (n,), "typestr": dtype.str, "data": (ptr, False),
                                                 "version": 3, "strides": None}

        from . import _lib

        def fn(ptr, n, dtype):
            # the collective is ordered on the library's stream: NCCL waits
            # for the deposit queued there, and the library's next kernels
            # wait for NCCL; the host does not wait
            ptr_s = _lib.lib().sb2_allreduce_stream()
            st = torch.cuda.ExternalStream(ptr_s) if ptr_s else torch.cuda.default_stream()
            with torch.cuda.stream(st):
                t = torch.as_tensor(_Dev(ptr, n, dtype), device="cuda")
                dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    propagator.set_allreduce(fn, on_host=on_host, typed=True)
    return propagator
