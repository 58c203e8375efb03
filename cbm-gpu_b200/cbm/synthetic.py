"""Seeded synthetic graphs that stand in for the reference's datasets.

The reference benchmarks on SNAP / SuiteSparse / OGB graphs loaded through
PyG (benchmark/utilities.py:92-199).  None of those datasets (nor PyG) exist
here, so every workload is generated from a numpy ``Generator(PCG64(seed))``
with the shapes, degree laws and near-duplicate structure of the five
workloads this library is measured on:

* ``community``  N nodes in communities; each node links to ``k_in`` distinct
  same-community nodes and ``k_out`` uniform-random nodes.
* ``chung_lu``   power-law expected degrees w_i ~ i^(-1/(gamma-1)) scaled to a
  mean degree and capped at sqrt(sum w) (the Chung-Lu admissibility bound);
  M = sum(w)/2 edges with both endpoints drawn proportionally to w.
* ``near_duplicates`` replaces a fraction of rows by copies of uniformly
  chosen template rows in which a fraction of the entries is flipped (each
  template entry dropped with that probability and as many uniform-random
  columns added), which is what gives CBM its compression.

Every generator returns a coalesced, symmetric ``edge_index`` (int32 [2, nnz],
sorted by (row, col)) with no self-loops, exactly the input the reference's
``cbm4*`` constructors take (cbm/cbm4mm.py:9).
"""
from __future__ import annotations

import math

import numpy as np

__all__ = [
    "coalesce_symmetric",
    "community_graph",
    "chung_lu_graph",
    "near_duplicates",
    "workload",
    "WORKLOADS",
]


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def coalesce_csr(rows, cols, n, symmetrize=True, drop_self=True):
    """COO -> CSR (int64 ptr, int32 sorted unique columns) by the library's
    native coalescer (cbm_coalesce)."""
    import ctypes as C

    from . import _lib

    lib = _lib.load()
    r = np.ascontiguousarray(rows, dtype=np.int32)
    c = np.ascontiguousarray(cols, dtype=np.int32)
    ptr = np.empty(n + 1, dtype=np.int64)
    out = np.empty(max(1, r.size * (2 if symmetrize else 1)), dtype=np.int32)
    nnz = C.c_int64(0)
    flags = (_lib.COALESCE_SYMMETRIZE if symmetrize else 0) | (_lib.COALESCE_DROP_SELF if drop_self else 0)
    _lib.check(lib.cbm_coalesce(r.ctypes.data, c.ctypes.data, r.size, n, flags, ptr.ctypes.data, out.ctypes.data,
                                C.byref(nnz)), "cbm_coalesce")
    return ptr, out[: nnz.value]


def coalesce_symmetric(rows, cols, n):
    """A | A^T with self-loops removed; returns int32 [2, nnz] sorted by (row, col)."""
    ptr, col = coalesce_csr(rows, cols, n)
    out = np.empty((2, col.size), dtype=np.int32)
    out[0] = np.repeat(np.arange(n, dtype=np.int32), np.diff(ptr))
    out[1] = col
    return out


def community_graph(n, community_size, k_in, k_out, seed=None, rng=None):
    """Communities of ``community_size``: k_in distinct in-community links, k_out uniform links."""
    rng = rng if rng is not None else _rng(seed)
    rows, cols = [], []
    node = np.arange(n, dtype=np.int64)
    comm_start = (node // community_size) * community_size
    comm_len = np.minimum(comm_start + community_size, n) - comm_start
    if k_in > 0 and community_size > 1:
        # k_in distinct others inside the community: rank random keys per node
        width = community_size - 1
        keys = rng.random((n, width))
        # positions past the (possibly short) last community are invalid
        valid = np.arange(width)[None, :] < (comm_len - 1)[:, None]
        keys[~valid] = 2.0
        k = min(k_in, width)
        pick = np.argpartition(keys, k - 1, axis=1)[:, :k] if k < width else np.tile(np.arange(width), (n, 1))
        pick_valid = np.take_along_axis(valid, pick, axis=1)
        local = node - comm_start
        other = pick + (pick >= local[:, None])  # skip the node itself
        dst = comm_start[:, None] + other
        src = np.broadcast_to(node[:, None], dst.shape)
        rows.append(src[pick_valid])
        cols.append(dst[pick_valid])
    if k_out > 0 and n > 1:
        r = rng.integers(0, n - 1, size=(n, k_out))
        r = r + (r >= node[:, None])
        rows.append(np.repeat(node, k_out))
        cols.append(r.reshape(-1))
    return coalesce_symmetric(np.concatenate(rows), np.concatenate(cols), n)


def chung_lu_weights(n, exponent, mean_degree):
    """Expected degrees w_i ~ i^(-1/(gamma-1)), mean ``mean_degree``, capped at sqrt(sum w)."""
    i = np.arange(1, n + 1, dtype=np.float64)
    w = i ** (-1.0 / (exponent - 1.0))
    w *= mean_degree / w.mean()
    cap = math.sqrt(w.sum())
    return np.minimum(w, cap)


def chung_lu_graph(n, exponent, mean_degree, seed=None, rng=None):
    rng = rng if rng is not None else _rng(seed)
    w = chung_lu_weights(n, exponent, mean_degree)
    m = int(round(w.sum() / 2.0))
    p = w / w.sum()
    cdf = np.cumsum(p)
    cdf[-1] = 1.0
    u = np.searchsorted(cdf, rng.random(m), side="right")
    v = np.searchsorted(cdf, rng.random(m), side="right")
    # a random relabelling so that hubs are not all at low ids
    perm = rng.permutation(n)
    return coalesce_symmetric(perm[u], perm[v], n)


def _csr(edge_index, n):
    rows = edge_index[0].astype(np.int64)
    cols = edge_index[1].astype(np.int64)
    ptr = np.zeros(n + 1, dtype=np.int64)
    ptr[1:] = np.cumsum(np.bincount(rows, minlength=n))
    return ptr, cols


def near_duplicates(edge_index, n, fraction, flip, seed=None, rng=None):
    """Replace ``fraction`` of the rows by flipped copies of template rows, then symmetrise."""
    rng = rng if rng is not None else _rng(seed)
    ptr, cols = _csr(edge_index, n)
    rows_all = edge_index[0].astype(np.int64)
    n_copy = int(round(fraction * n))
    perm = rng.permutation(n)
    copies = np.sort(perm[:n_copy])
    templates_pool = perm[n_copy:]
    templates = templates_pool[rng.integers(0, templates_pool.size, size=n_copy)]
    is_copy = np.zeros(n, dtype=bool)
    is_copy[copies] = True
    # rows that are not copies keep their entries
    keep = ~is_copy[rows_all]
    base_r = rows_all[keep]
    base_c = cols[keep]
    # copied entries: the template's row, each entry dropped with probability ``flip``
    tlen = ptr[templates + 1] - ptr[templates]
    total = int(tlen.sum())
    owner = np.repeat(np.arange(n_copy), tlen)
    start = np.repeat(ptr[templates], tlen)
    offs = np.arange(total) - np.repeat(np.cumsum(tlen) - tlen, tlen)
    c_cols = cols[start + offs]
    c_rows = copies[owner]
    drop = rng.random(total) < flip
    n_drop = np.bincount(owner[drop], minlength=n_copy)
    c_rows, c_cols = c_rows[~drop], c_cols[~drop]
    # as many uniform-random columns added as were dropped
    add_owner = np.repeat(np.arange(n_copy), n_drop)
    a_rows = copies[add_owner]
    a_cols = rng.integers(0, n, size=add_owner.size)
    r = np.concatenate([base_r, c_rows, a_rows])
    c = np.concatenate([base_c, c_cols, a_cols])
    return coalesce_symmetric(r, c, n)


# The five workloads: (name, builder).  Sizes, laws and seeds are the ones the
# bench and the parity tests use.
def _w_powerlaw(n, exponent, mean, frac, flip, seed):
    rng = _rng(seed)
    ei = chung_lu_graph(n, exponent, mean, rng=rng)
    return near_duplicates(ei, n, frac, flip, rng=rng)


WORKLOADS = {
    # plain A.X, fp32, alpha 0
    "community-4096": dict(n=4096, alpha=0, cols=64, seed=0,
                           build=lambda: community_graph(4096, 64, 12, 4, seed=0)),
    # D^-1/2 A D^-1/2 X, fp32, alpha 8
    "powerlaw-1m": dict(n=1_000_000, alpha=8, cols=256, seed=1,
                        build=lambda: _w_powerlaw(1_000_000, 2.1, 20.0, 0.30, 0.10, 1)),
    # A D^-1/2 X, bf16 X, alpha 16
    "powerlaw-2.4m": dict(n=2_400_000, alpha=16, cols=128, seed=2,
                          build=lambda: _w_powerlaw(2_400_000, 2.3, 50.0, 0.40, 0.05, 2)),
    # 2-layer GCN graph
    "powerlaw-170k": dict(n=170_000, alpha=0, cols=128, seed=3,
                          build=lambda: _w_powerlaw(170_000, 2.1, 14.0, 0.25, 0.10, 3)),
}


def workload(name):
    """Return (edge_index int32 [2, nnz], n, spec) for a named workload."""
    spec = WORKLOADS[name]
    ei = spec["build"]()
    return ei, spec["n"], spec


def batch_graphs(count=512, n_lo=1000, n_hi=64000, deg_lo=8.0, deg_hi=40.0, seed=4):
    """Many independent community graphs of log-uniform size and uniform mean degree.

    Community size 64 as in the 4096-node workload; a node gets
    round(0.75 * deg / 2) in-community links and the rest uniform, so that the
    symmetrised mean degree is close to ``deg``.
    """
    rng = _rng(seed)
    sizes = np.exp(rng.uniform(math.log(n_lo), math.log(n_hi), size=count)).astype(np.int64)
    degs = rng.uniform(deg_lo, deg_hi, size=count)
    graphs = []
    for n_i, d_i in zip(sizes, degs):
        k_total = max(1, int(round(d_i / 2.0)))
        k_in = max(1, int(round(0.75 * k_total)))
        k_out = max(0, k_total - k_in)
        graphs.append((community_graph(int(n_i), 64, k_in, k_out, rng=rng), int(n_i)))
    return graphs
