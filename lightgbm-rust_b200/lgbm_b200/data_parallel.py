"""Reductions over torch.distributed ranks for the data-parallel learner
(Learner.set_data_parallel): the learner hands over a buffer in its own
device memory; these reduce it in place over every rank of the process group.

- `torch_allreduce_nccl`: the buffer itself is reduced by NCCL (one GPU per
  rank; NVLink / NVSwitch between the GPUs).
- `torch_allreduce_host`: the buffer goes through host memory and the
  group's CPU backend (gloo); it works whatever the devices, one GPU shared by
  several ranks included.
"""
import torch
import torch.distributed as dist

from . import _lib as L

_DTYPES = {L.DT_INT64: ("<i8", torch.int64), L.DT_FLOAT64: ("<f8", torch.float64), L.DT_INT32: ("<i4", torch.int32)}
_OPS = {L.OP_SUM: dist.ReduceOp.SUM, L.OP_MAX: dist.ReduceOp.MAX}


class _DeviceBuffer:
    """A view of `count` values at device address `ptr` (no copy)."""

    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (ptr, False), "version": 3}


def _view(ptr, count, dtype, device):
    typestr, _ = _DTYPES[dtype]
    return torch.as_tensor(_DeviceBuffer(ptr, count, typestr), device=device)


def torch_allreduce_host(device, group=None):
    """A reduction through host memory on the process group's backend."""

    def allreduce(ptr, count, dtype, op):
        t = _view(ptr, count, dtype, device)
        h = t.cpu()
        dist.all_reduce(h, op=_OPS[op], group=group)
        t.copy_(h)
        torch.cuda.synchronize(device)

    return allreduce


def torch_allreduce_nccl(device, group=None):
    """A reduction of the device buffer itself by NCCL."""

    def allreduce(ptr, count, dtype, op):
        t = _view(ptr, count, dtype, device)
        dist.all_reduce(t, op=_OPS[op], group=group)
        torch.cuda.synchronize(device)

    return allreduce
