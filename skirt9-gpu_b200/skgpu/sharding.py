"""Sharding of a primary-emission segment over ranks (one process per GPU).

Histories are independent and every tally is additive, so ranks split a segment into contiguous
history ranges and the segment's tallies are the sum over ranks: the reference does this sum at the
end of a segment (FluxRecorder::calibrateAndWrite's ProcessManager::sumToRoot,
SKIRT/core/FluxRecorder.cpp:876-885, and MediumSystem::communicateRadiationField,
SKIRT/core/MediumSystem.cpp:2524-2547). Here the sum is one all-reduce over the ranks:

  allreduce_device_tallies  in place on the library's device tally buffers (NCCL over NVLink), after
                            which any rank fetches the segment's tallies;
  allreduce_results         on fetched host tallies (any backend, e.g. gloo on CPU).
"""
import numpy as np


def history_range(rank, world, n):
    """Contiguous share of [0, n) for `rank` (the last rank takes the remainder)."""
    per = n // world
    first = rank * per
    return first, (n - first if rank == world - 1 else per)


class _DeviceArray:
    """A device FP64 array of the library exposed through __cuda_array_interface__, so that torch
    wraps it without a copy."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 2}


def device_tally_tensors(be, device):
    """torch views of the context's device tally buffers (no copy)."""
    import torch
    from . import abi
    return [torch.as_tensor(_DeviceArray(p, n), device=device) for p, n in abi.tally_buffers(be) if n]


def allreduce_device_tallies(be, device, group=None):
    """Sums the device tallies of every rank in place (one all-reduce per buffer, in the same order on
    every rank); returns the bytes reduced per rank. Every rank must call it at the same point of its
    segment."""
    import torch
    import torch.distributed as dist
    tensors = device_tally_tensors(be, device)
    torch.cuda.synchronize(device)  # the library's stream has finished the segment
    for t in tensors:
        dist.all_reduce(t, group=group)
    torch.cuda.synchronize(device)
    return sum(8 * t.numel() for t in tensors)


def _result_arrays(res):
    arrays = []
    for ins in res.instruments:
        for key in ("total", "stats", "components"):
            if ins.get(key) is not None:
                arrays.append(ins[key])
    if res.rf is not None:
        arrays.append(res.rf)
    return arrays


def allreduce_results(res, group=None):
    """Sums fetched host tallies (a Results: every instrument's total, statistics and components,
    and the radiation field) over the ranks in place, through one flat FP64 all-reduce."""
    import torch
    import torch.distributed as dist
    arrays = _result_arrays(res)
    flat = torch.from_numpy(np.concatenate([np.asarray(a, np.float64).ravel() for a in arrays]))
    dist.all_reduce(flat, group=group)
    off = 0
    out = flat.numpy()
    for a in arrays:
        a[...] = out[off:off + a.size].reshape(a.shape)
        off += a.size
    return res
