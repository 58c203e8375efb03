"""Tree shards (cbm.shard): whole trees of the CBM forest per rank, X rows
all-gathered, Y row-owned.  On CPU: the split keeps every tree on one rank and
is balanced; every rank's rows, multiplied by the oracle on the rank's own
structure, equal the same rows of the unsplit product bit for bit; and over
world_size-2 gloo ranks, X assembled by the all-gather composes the product.
"""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from conftest import near_dup_graph


def _structure(n=1500, seed=7):
    from cbm import cbm_mkl_cpp

    ei = near_dup_graph(n, seed=seed, deg=10)
    return cbm_mkl_cpp.build(ei[0], ei[1], n, 0), n


def _dad_values(s, n):
    d = np.diff(s.csr_ptr).astype(np.float32)  # any positive multipliers will do
    m = (1.0 / np.sqrt(np.maximum(d, 1.0))).astype(np.float32)
    rows = np.repeat(np.arange(n), np.diff(s.csr_ptr))
    return ((s.csr_val * m[s.csr_col]) * m[rows]).astype(np.float32), m


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_tree_owner_keeps_trees_whole_and_balances(world):
    from cbm.shard import tree_owner, tree_roots

    s, n = _structure()
    owner = tree_owner(s.parent, s.csr_ptr, world)
    root = tree_roots(s.parent)
    assert np.array_equal(owner, owner[root])  # a tree's rows share its root's rank
    assert np.all(owner[s.src] == owner[s.dst])
    cost = np.bincount(owner, weights=np.diff(s.csr_ptr) + 1.0, minlength=world)
    biggest = np.bincount(root, weights=np.diff(s.csr_ptr) + 1.0).max()
    assert cost.max() - cost.min() <= biggest  # greedy: within one tree's cost
    assert np.array_equal(owner, tree_owner(s.parent, s.csr_ptr, world))


@pytest.mark.parametrize("world", [2, 5])
@pytest.mark.parametrize("op", ["ax", "dad"])
def test_tree_shards_compose_the_product(world, op):
    from cbm.shard import TreeShard, tree_owner
    from oracle import oracle

    s, n = _structure()
    x = np.random.default_rng(3).standard_normal((n, 24)).astype(np.float32)
    owner = tree_owner(s.parent, s.csr_ptr, world)
    if op == "ax":
        full = oracle.spmm_update(s.csr_ptr, s.csr_col, s.csr_val, x, s.branches, s.src, s.dst)
        vals, m = s.csr_val, None
    else:
        vals, m = _dad_values(s, n)
        full = oracle.spmm_fused_update(s.csr_ptr, s.csr_col, vals, x, s.branches, s.src, s.dst, m, gpu_order=True)
    y = np.full_like(full, np.nan)
    for r in range(world):
        sh = TreeShard(s, owner, r, values=vals)
        assert sh.n_cols == n and sh.row_ptr[-1] == sh.col.size
        if op == "ax":
            part = oracle.spmm_update(sh.row_ptr, sh.col, sh.val, x, sh.branches, sh.src, sh.dst)
        else:
            part = oracle.spmm_fused_update(sh.row_ptr, sh.col, sh.val, x, sh.branches, sh.src, sh.dst,
                                            m[sh.rows], gpu_order=True)
        y[sh.rows] = part
    assert np.array_equal(y, full)


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _worker(rank, world, port, results):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    repo = os.path.dirname(here)
    for p in (os.path.join(repo, "cbm-gpu_b200"), repo, here):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from cbm.shard import TreeShard, gather_rows, tree_owner
        from oracle import oracle

        s, n = _structure(900, seed=9)
        x_full = np.random.default_rng(5).standard_normal((n, 16)).astype(np.float32)
        owner = tree_owner(s.parent, s.csr_ptr, world)
        sh = TreeShard(s, owner, rank)
        # each rank starts from its own rows of X only
        x = gather_rows(torch.from_numpy(x_full[sh.rows]), owner, rank, world).numpy()
        y_local = oracle.spmm_update(sh.row_ptr, sh.col, sh.val, x, sh.branches, sh.src, sh.dst)
        parts = [None] * world
        dist.all_gather_object(parts, (sh.rows, y_local))
        if rank == 0:
            full = oracle.spmm_update(s.csr_ptr, s.csr_col, s.csr_val, x_full, s.branches, s.src, s.dst)
            y = np.full_like(full, np.nan)
            for rows, part in parts:
                y[rows] = part
            results.put(("ok", bool(np.array_equal(x, x_full)), bool(np.array_equal(y, full))))
        else:
            results.put(("rank", rank))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_tree_shards_with_x_all_gather():
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = [q.get() for _ in range(2)]
    ok = next(g for g in got if g[0] == "ok")
    assert ok[1], "X assembled by the all-gather differs"
    assert ok[2], "tree shards do not compose to the unsplit product"


@pytest.mark.gpu
def test_tree_shard_plans_on_the_gpu_equal_the_full_product():
    """Each shard as a rectangular plan (its rows x all columns) on the GPU:
    the VALUES ops with prepared D^-1/2 A D^-1/2 values and per-row
    multipliers give the full cbm4dad product's rows bit for bit."""
    from cbm.cbm4dad import cbm4dad
    from cbm.plan import Plan
    from cbm.shard import TreeShard, tree_owner

    n = 3000
    ei = near_dup_graph(n, seed=12, deg=12)
    a = cbm4dad(torch.from_numpy(ei), torch.ones(ei.shape[1]), alpha=0)
    from cbm import cbm_mkl_cpp

    s = cbm_mkl_cpp.build(ei[0], ei[1], n, 0)
    vals = a.deltas.values().cpu().numpy()
    m = a.D.cpu().numpy()
    x = torch.randn(n, 64, device="cuda")
    y_full = torch.empty_like(x)
    a.matmul(x, y_full)
    owner = tree_owner(s.parent, s.csr_ptr, 3)
    y = torch.full_like(x, float("nan"))
    for r in range(3):
        sh = TreeShard(s, owner, r, values=vals)
        p = Plan(sh.row_ptr, sh.col, sh.val, sh.n_rows, sh.n_cols, sh.branches, sh.src, sh.dst,
                 multipliers=m[sh.rows], host=True)
        part = torch.empty(sh.n_rows, 64, device="cuda")
        p.matmul("values_ratio", x, part)
        p.check_device()
        y[torch.from_numpy(sh.rows).cuda()] = part
    assert torch.equal(y, y_full)
