"""Multi-GPU counting of one field: z-slab shards, one process per GPU, counts summed by all-reduce.

The pattern counts are a sum over cells, and a cell needs two adjacent planes, so a field of Z
planes splits into slabs of cell planes; every rank reads its cell planes plus the next plane
(one halo plane shared with the following rank), counts its slab alone, and one all-reduce of
the K x 256 uint64 counts (NCCL over NVLink for CUDA tensors, gloo for CPU tensors) combines
them. No field data crosses between GPUs; the halo plane is read by both neighbours.
The original library counts one field on one GPU (mkfCUDA.cu:12-61); this is the sharded form of
the same sum.
"""
from __future__ import annotations

from typing import Callable

import numpy as np


def slab_cells(Z: int, world: int, rank: int) -> tuple[int, int]:
    """Cell planes [c0, c1) of `rank`'s share of a Z-plane field (cell plane z joins planes z and
    z + 1). Shares differ by at most one plane; ranks beyond the cell count get empty shares."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    cells = max(Z - 1, 0)
    base, rem = divmod(cells, world)
    c0 = rank * base + min(rank, rem)
    return c0, c0 + base + (1 if rank < rem else 0)


def slab_planes(Z: int, world: int, rank: int) -> tuple[int, int]:
    """Field planes [z0, z1) that `rank` reads: its cell planes plus one halo plane (z1 - z0 is 0
    for an empty share)."""
    c0, c1 = slab_cells(Z, world, rank)
    return (c0, c1 + 1) if c1 > c0 else (c0, c0)


def sharded_field_bpfd(slab, thresholds, mask=None, group=None, out=None, stream=None,
                       counter: Callable | None = None):
    """Pattern counts of a whole field from this rank's slab (planes `slab_planes(Z, world, rank)`
    of the field, as a (planes, Y, X) tensor). Every rank of `group` must call it with the same
    thresholds; the result, identical on every rank, is the (K, 256) int64 count tensor of the
    whole field.

    `counter(slab, thresholds, mask, out)` counts one slab into `out` (default: the CUDA kernel,
    `field_bpfd`; a CPU tensor needs an explicit counter)."""
    import torch
    import torch.distributed as dist

    from . import BMC_GT, field_bpfd

    if mask is None:
        mask = BMC_GT
    K = len(np.atleast_1d(np.asarray(thresholds, dtype=np.float64)))
    if out is None:
        out = torch.zeros((K, 256), dtype=torch.int64, device=slab.device)
    else:
        out.zero_()
    if slab.shape[0] >= 2:
        if counter is None:
            if slab.device.type != "cuda":
                raise ValueError("the default counter needs a CUDA slab")
            field_bpfd(slab, thresholds, mask, out=out, accumulate=True, stream=stream)
        else:
            counter(slab, thresholds, mask, out)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(out, op=dist.ReduceOp.SUM, group=group)
    return out
