"""Host logic of the multi-GPU form: one process per GPU.

Two splits of Y = op(A) X; the reference is single-GPU (cbm/cbm.cu has no
communication) and has no counterpart of either.

Column shards (``column_shard``): rank r owns the columns [c0, c1) of X and Y
and a full replica of the CBM structure, and computes Y[:, c0:c1] =
op(A) X[:, c0:c1] on its own GPU.  Nothing crosses NVLink on the data path;
the only collectives are the timing reduction (max over ranks) and barriers.

Tree shards (``tree_owner``, ``TreeShard``, ``gather_rows``): rank r owns
whole trees of the CBM forest (a root row and all its descendants, so every
tree edge stays on one rank) and their rows of Y, and holds only those rows'
delta entries and edges: the structure's memory divides by the rank count,
which column shards do not.  Its rows gather X rows of any node, so X is
first assembled on every rank from each rank's own rows (``gather_rows``, an
all-gather over NCCL); Y stays row-owned and needs no reduction.  Each rank's
product is bit-identical to the same rows of the unsplit product.
"""
from __future__ import annotations

import os

import torch

import numpy as np

__all__ = ["column_shard", "max_over_ranks", "build_once", "tree_roots", "tree_owner", "TreeShard", "gather_rows"]


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


def tree_roots(parent):
    """Root of every node's tree; ``parent[v] == len(parent)`` marks a root (the
    virtual root's child)."""
    parent = np.asarray(parent, dtype=np.int64)
    n = parent.size
    r = np.where(parent == n, np.arange(n), parent)
    while True:  # pointer jumping: depth halves every step
        nxt = r[r]
        if np.array_equal(nxt, r):
            return r
        r = nxt


def tree_owner(parent, row_ptr, world):
    """Owner rank of every row: whole trees, largest first (cost: delta entries
    plus one per row) to the least-loaded rank, ties to the lower rank and the
    lower root id, so every rank computes the same split."""
    if world < 1:
        raise ValueError("world must be at least 1")
    parent = np.asarray(parent, dtype=np.int64)
    n = parent.size
    root = tree_roots(parent)
    cost = np.bincount(root, weights=np.diff(np.asarray(row_ptr, dtype=np.int64)) + 1.0, minlength=n)
    trees = np.flatnonzero(np.bincount(root, minlength=n))
    order = trees[np.argsort(-cost[trees], kind="stable")]
    load = np.zeros(world)
    tree_rank = np.zeros(n, dtype=np.int32)
    for t in order:
        r = int(np.argmin(load))
        tree_rank[t] = r
        load[r] += cost[t]
    return tree_rank[root]


class TreeShard:
    """Rank ``rank``'s part of a CBM structure under ``owner``: its rows in
    increasing global id (local row i is global row ``rows[i]``), their delta
    entries (global column ids) and the tree edges among them, in their BFS
    order with the branch offsets recomputed.  ``values`` (default: the
    structure's +-1) are per entry of the whole structure."""

    def __init__(self, s, owner, rank, values=None):
        owner = np.asarray(owner)
        n = owner.size
        self.rows = np.flatnonzero(owner == rank).astype(np.int64)
        local = np.full(n, -1, dtype=np.int64)
        local[self.rows] = np.arange(self.rows.size)
        ptr = np.asarray(s.csr_ptr, dtype=np.int64)
        lens = ptr[self.rows + 1] - ptr[self.rows]
        self.row_ptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
        take = (np.repeat(ptr[self.rows] - self.row_ptr[:-1], lens) + np.arange(int(lens.sum()))).astype(np.int64)
        vals = s.csr_val if values is None else np.asarray(values, dtype=np.float32)
        self.col = np.asarray(s.csr_col)[take].astype(np.int32)
        self.val = vals[take].astype(np.float32)
        src, dst = np.asarray(s.src, dtype=np.int64), np.asarray(s.dst, dtype=np.int64)
        mine = owner[dst] == rank
        if np.any(owner[src[mine]] != rank):
            raise RuntimeError("a tree edge crosses ranks: owner must keep whole trees together")
        self.src = local[src[mine]].astype(np.int32)
        self.dst = local[dst[mine]].astype(np.int32)
        br = np.asarray(s.branches, dtype=np.int64)
        lens = np.diff(br)
        starts = br[:-1][lens > 0]
        kept = lens[lens > 0][owner[dst[starts]] == rank] if starts.size else np.zeros(0, dtype=np.int64)
        self.branches = np.concatenate([[0], np.cumsum(kept)]).astype(np.int32)
        if int(self.branches[-1]) != self.src.size:
            raise RuntimeError("branch offsets do not cover this rank's edges")
        self.n_rows = int(self.rows.size)
        self.n_cols = n


def gather_rows(x_local, owner, rank, world, group=None):
    """X [n, C] on every rank from each rank's own rows (``x_local``: the rows
    owner == rank, in increasing id): one all-gather of equal-sized padded
    blocks, then every block scattered to its rows."""
    import torch.distributed as dist

    owner = np.asarray(owner)
    counts = np.bincount(owner, minlength=world)
    pad = int(counts.max()) if counts.size else 0
    if x_local.shape[0] != counts[rank]:
        raise ValueError(f"rank {rank} holds {x_local.shape[0]} rows, owns {counts[rank]}")
    block = torch.zeros((pad,) + tuple(x_local.shape[1:]), dtype=x_local.dtype, device=x_local.device)
    block[: x_local.shape[0]] = x_local
    out = torch.empty((world * pad,) + tuple(x_local.shape[1:]), dtype=x_local.dtype, device=x_local.device)
    if world > 1:
        dist.all_gather_into_tensor(out, block, group=group)
    else:
        out.copy_(block)
    x = torch.empty((owner.size,) + tuple(x_local.shape[1:]), dtype=x_local.dtype, device=x_local.device)
    for r in range(world):
        rows = torch.from_numpy(np.flatnonzero(owner == r)).to(x_local.device)
        x.index_copy_(0, rows, out[r * pad: r * pad + int(counts[r])])
    return x
