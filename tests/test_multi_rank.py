"""Multi-GPU form, host side: column shards over world_size-2 ``gloo`` ranks on CPU.

Each rank owns a contiguous block of X's and Y's columns and a full replica of
the CBM structure; no data crosses ranks between products.  Here each rank
computes its shard with the CPU oracle (the GPU kernels are exercised by the
-m gpu tests), the shards are gathered, and rank 0 checks that they compose
to the unsharded product bit for bit.  Also covered: the shard bounds, the
max-over-ranks timing reduction and the rank-0 file cache behind a barrier.
"""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("total,world", [(256, 1), (512, 2), (1024, 8), (130, 4), (3, 2), (0, 2)])
def test_column_shard_bounds_tile_the_columns(total, world):
    from cbm.shard import column_shard

    bounds = [column_shard(total, r, world) for r in range(world)]
    assert bounds[0][0] == 0 and bounds[-1][1] == total
    for (a0, a1), (b0, b1) in zip(bounds, bounds[1:]):
        assert a1 == b0 and a0 <= a1
    for c0, _ in bounds:
        assert c0 % 4 == 0 or c0 == total
    if total % (4 * world) == 0:
        assert len({c1 - c0 for c0, c1 in bounds}) == 1


def test_column_shard_rejects_bad_ranks():
    from cbm.shard import column_shard

    with pytest.raises(ValueError):
        column_shard(256, 2, 2)
    with pytest.raises(ValueError):
        column_shard(256, 0, 0)


def _worker(rank, world, port, tmpdir, results):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    repo = os.path.dirname(here)
    for p in (os.path.join(repo, "cbm-gpu_b200"), repo, here):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from cbm import cbm_mkl_cpp
        from cbm.shard import build_once, column_shard, max_over_ranks
        from conftest import near_dup_graph
        from oracle import oracle

        # the graph is made once by rank 0 and read by every rank
        path = os.path.join(tmpdir, "graph.npz")

        def make(p):
            with open(p, "wb") as f:
                np.savez(f, ei=near_dup_graph(600, seed=5, deg=10))

        ei = np.load(build_once(path, make, rank))["ei"]
        n = int(ei.max()) + 1
        s = cbm_mkl_cpp.build(ei[0], ei[1], n, 0)
        deg = np.diff(s.csr_ptr).astype(np.float32)
        total = 96
        x = np.random.default_rng(11).standard_normal((n, total)).astype(np.float32)
        c0, c1 = column_shard(total, rank, world)
        args = (s.csr_ptr, s.csr_col, s.csr_val)
        tree = (s.branches, s.src, s.dst)
        y_shard = oracle.spmm_update(*args, np.ascontiguousarray(x[:, c0:c1]), *tree)
        shards = [None] * world
        dist.all_gather_object(shards, (c0, c1, y_shard))
        t = max_over_ranks(1.5 + rank)
        if rank == 0:
            full = oracle.spmm_update(*args, x, *tree)
            y = np.concatenate([sh[2] for sh in sorted(shards, key=lambda q: q[0])], axis=1)
            results.put(("ok", bool(np.array_equal(y, full)), t, deg.size == n))
        else:
            results.put(("rank", rank, t))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_compose_the_product():
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    with tempfile.TemporaryDirectory() as tmpdir:
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, tmpdir, q)) for r in range(2)]
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
    other = next(g for g in got if g[0] == "rank")
    assert ok[1], "column shards do not compose to the unsharded product"
    assert ok[2] == 2.5 and other[2] == 2.5, "max over ranks"
    assert ok[3]


def test_max_over_ranks_single_process():
    from cbm.shard import max_over_ranks

    assert max_over_ranks(3.25) == 3.25
