"""LSH clustering (benchmark/clustering_gpu.py:86-183) and the clustered CBM.

CPU: the clusters partition the non-empty rows, respect the size bound, and
match a direct restatement of the reference's loop on a small graph; the
clustered construction equals building each cluster's CBM separately (the
reference's cbm4mm per cluster) and restricts every parent to its cluster.
GPU: the clustered CBM's product equals the oracle's on its structure and
the FP64 product of A."""
import numpy as np
import pytest
import torch

from conftest import near_dup_graph


def _reference_loop(edge_index, n, max_cluster_size, num_hashes):
    """The reference's loop, restated with numpy (no merge)."""
    rows_of = [[] for _ in range(n)]
    for r, c in zip(edge_index[0], edge_index[1]):
        rows_of[r].append(c)
    rows_of = [sorted(set(x)) for x in rows_of]
    opened = [np.array([r for r in range(n) if rows_of[r]], dtype=np.int64)]
    closed = []
    while opened:
        rows = opened.pop()
        counts = np.zeros(n)
        for r in rows:
            counts[rows_of[r]] += 1
        dist = np.abs(counts - rows.size / 2.0)
        hashes = np.sort(np.argsort(dist, kind="stable")[:num_hashes])
        bit = {int(h): 1 << j for j, h in enumerate(hashes)}
        fp = np.array([sum(bit.get(c, 0) for c in rows_of[r]) for r in rows])
        groups = [rows[fp == u] for u in np.unique(fp)]
        if len(groups) == 1:
            closed.append(groups[0])
            continue
        for g in groups:
            (closed if g.size <= max_cluster_size else opened).append(g)
    return closed


def test_lsh_clusters_match_the_restated_loop():
    from cbm.cluster import lsh_clusters

    ei = near_dup_graph(600, seed=12)
    got = lsh_clusters(ei, 600, max_cluster_size=80, num_hashes=4, device="cpu", merge=False)
    ref = _reference_loop(ei, 600, 80, 4)
    key = lambda cs: sorted(tuple(sorted(c.tolist())) for c in cs)  # noqa: E731
    assert key(got) == key(ref)


@pytest.mark.parametrize("max_size", [50, 200, 1000])
def test_merged_clusters_partition_rows(max_size):
    from cbm.cluster import lsh_clusters

    ei = near_dup_graph(1500, seed=4)
    raw = lsh_clusters(ei, 1500, max_cluster_size=max_size, device="cpu", merge=False)
    cl = lsh_clusters(ei, 1500, max_cluster_size=max_size, device="cpu")
    allrows = np.sort(np.concatenate(cl))
    assert np.array_equal(allrows, np.unique(ei[0]))
    # merging never makes a cluster larger than the bound (only groups that
    # could not be split may exceed it, and those are left as they are)
    big = sorted(c.size for c in raw if c.size > max_size)
    assert sorted(c.size for c in cl if c.size > max_size) == big
    assert len(cl) <= len(raw)


def test_clustered_structure_equals_per_cluster_builds():
    from cbm import cbm_mkl_cpp
    from cbm.cluster import cluster_ids, lsh_clusters

    n = 900
    ei = near_dup_graph(n, seed=6)
    cl = lsh_clusters(ei, n, max_cluster_size=150, device="cpu")
    ids = cluster_ids(cl, n)
    s = cbm_mkl_cpp.build(ei[0], ei[1], n, 0, cluster=ids)
    par = s.parent
    inner = par != n
    assert np.all(ids[par[inner]] == ids[inner]), "a parent outside its child's cluster"
    total = 0
    for c in cl:
        keep = np.isin(ei[0], c)
        sc = cbm_mkl_cpp.build(ei[0][keep], ei[1][keep], n, 0)
        total += sc.csr_col.size
    assert s.csr_col.size == total  # the same forests, so the same delta count
    assert s.tree_cost == total


@pytest.mark.gpu
def test_clustered_cbm_product():
    from cbm.cbm4dad import cbm4dad
    from cbm.cluster import cluster_ids, lsh_clusters
    from oracle import oracle

    n = 3000
    ei = near_dup_graph(n, seed=15, deg=12)
    cl = lsh_clusters(ei, n, max_cluster_size=400)
    a = cbm4dad(torch.from_numpy(ei), torch.ones(ei.shape[1]), alpha=0, cluster=cluster_ids(cl, n))
    x = torch.randn(n, 64, device="cuda")
    y = torch.empty_like(x)
    a.matmul(x, y)
    a.plan.check_device()
    ref = oracle.spmm_fused_update(a.deltas.crow_indices().cpu().numpy(), a.deltas.col_indices().cpu().numpy(),
                                   a.deltas.values().cpu().numpy(), x.cpu().numpy(), a.mca_offset.cpu().numpy(),
                                   a.mca_src_idx.cpu().numpy(), a.mca_dst_idx.cpu().numpy(), a.D.cpu().numpy(),
                                   gpu_order=True)
    np.testing.assert_array_equal(y.cpu().numpy(), ref)
    ptr, idx = oracle.csr_from_edges(ei, n)
    d = 1.0 / np.sqrt(np.diff(ptr).astype(np.float64))
    y64 = oracle.dense_f64(ptr, idx, n, x.double().cpu().numpy(), rs=d, cs=d)
    assert np.abs(y.cpu().numpy() - y64).max() <= 1e-5 * np.abs(y64).max() + 1e-6
