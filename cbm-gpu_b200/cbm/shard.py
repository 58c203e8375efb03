"""Host logic of the multi-GPU form: one process per GPU, column shards.

The product Y = op(A) X splits by columns with no exchange: rank r owns the
columns [c0, c1) of X and Y and a full replica of the CBM structure, and
computes Y[:, c0:c1] = op(A) X[:, c0:c1] on its own GPU.  Nothing crosses
NVLink on the data path, so no collective runs between products; the only
collectives are the timing reduction (max over ranks) and the barriers around
the timed region.  The reference is single-GPU (cbm/cbm.cu has no
communication) and has no counterpart.
"""
from __future__ import annotations

import os

import torch

__all__ = ["column_shard", "max_over_ranks", "build_once"]


def column_shard(total_cols, rank, world, align=4):
    """Columns [c0, c1) of rank ``rank``: contiguous, balanced, boundaries on
    multiples of ``align`` (16-byte rows for the vector path) where possible."""
    if world < 1 or not 0 <= rank < world or total_cols < 0:
        raise ValueError(f"bad shard request: {total_cols} columns, rank {rank} of {world}")
    units = (total_cols + align - 1) // align
    u0 = units * rank // world
    u1 = units * (rank + 1) // world
    return min(u0 * align, total_cols), min(u1 * align, total_cols)


def max_over_ranks(value, device=None):
    """The maximum of a float over all ranks (the value itself with one process)."""
    if not (torch.distributed.is_available() and torch.distributed.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def build_once(path, make, rank):
    """Rank 0 writes ``make()``'s bytes to ``path`` (atomically) if absent; every
    rank waits at a barrier, then reads the file.  Returns the bytes' path."""
    if rank == 0 and not os.path.exists(path):
        tmp = f"{path}.tmp{os.getpid()}"
        make(tmp)
        os.replace(tmp, path)
    if torch.distributed.is_available() and torch.distributed.is_initialized():
        torch.distributed.barrier()
    if not os.path.exists(path):
        raise RuntimeError(f"{path} was not written by rank 0")
    return path
