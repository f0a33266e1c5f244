"""Particle sharding across ranks (one process per GPU).

The push/scatter shards by particles with no data-path exchange; the one real
exchange of a sharded PIC step is the node-density sum, done in place on the
device between mp_push_scatter and mp_compute_phi.  The field solve then runs
replicated on every rank from the same summed density (the dense Newton
factorization does not shard; each rank holds its own copy)."""
from __future__ import annotations

import numpy as np


def shard_range(n: int, rank: int, world: int) -> slice:
    """Contiguous, balanced share [lo, hi) of n particles for `rank`."""
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    hi = lo + base + (1 if rank < extra else 0)
    return slice(lo, hi)


class _CudaArray:
    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                         "strides": None, "stream": None}


def device_vector(ctx, name: str, device: int):
    """A torch view (no copy) of a context's FP64 device vector."""
    import torch
    ptr, n = ctx.device_buffer(name)
    return torch.as_tensor(_CudaArray(ptr, n), device=f"cuda:{device}")


def allreduce_density(ctx, device: int, group=None) -> None:
    """Sums the node density of all ranks in place (NCCL over NVLink on GPUs).
    mp_push_scatter has synchronised the context's stream before returning, so
    the density is complete; the all-reduce is waited for before the caller's
    next context call."""
    import torch
    import torch.distributed as dist
    t = device_vector(ctx, "den", device)
    dist.all_reduce(t, group=group)
    torch.cuda.current_stream(device).synchronize()


def allreduce_density_host(den: np.ndarray, group=None) -> np.ndarray:
    """The same reduction on a host array (gloo); used by the CPU tests of the
    sharded step."""
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(np.ascontiguousarray(den))
    dist.all_reduce(t, group=group)
    return t.numpy()
