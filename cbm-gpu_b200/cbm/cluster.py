"""LSH clustering of a matrix's rows and the clustered CBM built from it.

``lsh_clusters(edge_index, n)`` follows the reference's hierarchical
fingerprinting (benchmark/clustering_gpu.py:86-183):

1. The rows that hold entries form one open cluster.
2. For an open cluster of r rows, count each column over the cluster's rows.
   Take the ``num_hashes`` columns whose count is closest to r / 2 (the
   columns of highest entropy; ties go to the lower column id), in increasing
   column order. A row's fingerprint is the sum of 2^j over the chosen
   columns j it holds. Rows with equal fingerprints form a new cluster.
3. Clusters of at most ``max_cluster_size`` rows are closed; larger ones are
   opened again. A cluster that did not split at all is closed as it is
   (fingerprinting it again would give the same result forever).
4. The closed clusters are sorted by size and merged from both ends
   (:160-182): the smallest are appended to the current largest while the sum
   stays within ``max_cluster_size``.

The reference then builds one cbm4mm per cluster (:184-195).  Here a single
structure holds them all: ``cbm4mm(..., cluster=ids)`` (or
``cbm_mkl_cpp.build(..., cluster=ids)``) restricts each row's parent to its
own cluster, so the per-cluster forests share one plan and one launch.

The fingerprinting runs in torch on ``device`` (the GPU when there is one,
like the reference); it is set-up work, not part of the product.
"""
from __future__ import annotations

import numpy as np
import torch

__all__ = ["lsh_clusters", "merge_clusters", "cluster_ids", "clustered_stats"]


def _csr(edge_index, n, device):
    r = torch.as_tensor(np.asarray(edge_index[0]), dtype=torch.int64, device=device)
    c = torch.as_tensor(np.asarray(edge_index[1]), dtype=torch.int64, device=device)
    key = torch.unique(r * n + c)  # coalesced, sorted by (row, col)
    rows, cols = key // n, key % n
    ptr = torch.zeros(n + 1, dtype=torch.int64, device=device)
    ptr[1:] = torch.cumsum(torch.bincount(rows, minlength=n), 0)
    return ptr, cols


def _fingerprints(ptr, cols, rows, n, num_hashes):
    """Fingerprints of `rows` (int64 tensor) over the num_hashes columns whose
    count within these rows is closest to half their number."""
    starts, ends = ptr[rows], ptr[rows + 1]
    lens = ends - starts
    owner = torch.repeat_interleave(torch.arange(rows.numel(), device=rows.device), lens)
    pos = torch.arange(int(lens.sum()), device=rows.device) - torch.repeat_interleave(
        torch.cumsum(lens, 0) - lens, lens) + torch.repeat_interleave(starts, lens)
    ecols = cols[pos]
    counts = torch.bincount(ecols, minlength=n).to(torch.float64)
    dist = (counts - rows.numel() / 2.0).abs()
    # smallest distance, ties to the lower column id (a stable sort)
    order = torch.sort(dist, stable=True).indices
    hashes = torch.sort(order[:num_hashes]).values
    weight = torch.zeros(n, dtype=torch.int64, device=rows.device)
    weight[hashes] = 2 ** torch.arange(hashes.numel(), dtype=torch.int64, device=rows.device)
    fp = torch.zeros(rows.numel(), dtype=torch.int64, device=rows.device)
    fp.scatter_add_(0, owner, weight[ecols])
    return fp


def merge_clusters(clusters, max_cluster_size):
    """The reference's two-ended merge of size-sorted clusters
    (benchmark/clustering_gpu.py:160-182)."""
    cl = sorted(clusters, key=lambda c: c.size)
    if not cl:
        return []
    merged = []
    b, e = 0, len(cl) - 1
    cur = cl[e]
    while b < e:
        if cl[b].size + cur.size <= max_cluster_size:
            cur = np.concatenate([cl[b], cur])
            b += 1
        else:
            merged.append(cur)
            e -= 1
            cur = cl[e]
    merged.append(cur)
    return merged


def lsh_clusters(edge_index, n, max_cluster_size=100000, num_hashes=4, device=None, merge=True):
    """Row clusters (list of int64 numpy arrays of row ids) of the n x n binary
    matrix given by edge_index."""
    if device is None:
        device = torch.device("cuda" if torch.cuda.is_available() else "cpu")
    ptr, cols = _csr(edge_index, n, device)
    lens = ptr[1:] - ptr[:-1]
    opened = [torch.nonzero(lens > 0).flatten()]
    closed = []
    while opened:
        rows = opened.pop()
        fp = _fingerprints(ptr, cols, rows, n, num_hashes)
        uniq, inverse = torch.unique(fp, return_inverse=True)
        order = torch.argsort(inverse, stable=True)
        counts = torch.bincount(inverse, minlength=uniq.numel()).tolist()
        groups = torch.split(rows[order], counts)
        if len(groups) == 1:
            closed.append(groups[0])
            continue
        for g in groups:
            (closed if g.numel() <= max_cluster_size else opened).append(g)
    out = [g.cpu().numpy().astype(np.int64) for g in closed]
    return merge_clusters(out, max_cluster_size) if merge else out


def cluster_ids(clusters, n):
    """Cluster id of every row (int32 [n]); rows in no cluster (no entries) get
    ids of their own, after the clusters'."""
    ids = np.arange(len(clusters), len(clusters) + n, dtype=np.int64)
    for k, c in enumerate(clusters):
        ids[c] = k
    if ids.max(initial=0) >= 2 ** 31:
        raise RuntimeError("too many rows for int32 cluster ids")
    return ids.astype(np.int32)


def clustered_stats(edge_index, n, clusters, alpha=0):
    """The reference's report (benchmark/clustering_gpu.py:204-215): nonzeros
    of A, of the unclustered CBM's delta matrix and of the clustered one."""
    from . import cbm_mkl_cpp

    s0 = cbm_mkl_cpp.build(edge_index[0], edge_index[1], n, alpha)
    s1 = cbm_mkl_cpp.build(edge_index[0], edge_index[1], n, alpha, cluster=cluster_ids(clusters, n))
    return {"nnz_csr": int(s0.nnz_a), "nnz_cbm": int(s0.csr_col.size), "nnz_cbm_clustered": int(s1.csr_col.size),
            "clusters": len(clusters), "largest": int(max((c.size for c in clusters), default=0))}
