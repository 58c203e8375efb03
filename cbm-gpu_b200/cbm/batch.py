"""Batching form: many graphs (or clusters) of uneven size in one launch.

``cbm_batch(graphs, alpha, op)`` builds each graph's CBM on the host (in
parallel: one constructor call per graph on a thread pool; the calls release
the GIL) and packs them block-diagonally into one structure: rows, columns and
tree edges of graph g are offset by the number of nodes before it.  One plan
then serves the whole batch, so one persistent launch (one device work queue
over every graph's rows, tree levels ordered across graphs) computes all
products.  ``capture`` records that launch in a CUDA graph for replay.

The reference has no batched product; its LSH clustering
(benchmark/clustering_gpu.py:159-197) builds one cbm4mm per cluster and
multiplies them one by one.
"""
from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor

import numpy as np
import torch

from . import cbm_mkl_cpp
from .plan import Plan

__all__ = ["cbm_batch"]


class cbm_batch:  # noqa: N801 (named like the other operator classes)
    """Block-diagonal CBM of several graphs; products for all of them at once."""

    def __init__(self, graphs, alpha=0, op="ax", threads=None):
        """graphs: list of (edge_index int32 [2, nnz], n_nodes) pairs."""
        if op not in ("ax", "adx", "dadx"):
            raise ValueError(f"op must be ax, adx or dadx, not {op}")
        self.op = op
        sizes = [int(n) for _, n in graphs]
        self.sizes = sizes
        self.offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        total = int(self.offsets[-1])
        if total >= 2 ** 30:
            raise RuntimeError("a batch holds fewer than 2^30 nodes")

        def build(g):
            ei, n = g
            return cbm_mkl_cpp.build(np.ascontiguousarray(ei[0], dtype=np.int32),
                                     np.ascontiguousarray(ei[1], dtype=np.int32), int(n), alpha, n_threads=1)

        with ThreadPoolExecutor(max_workers=threads) as ex:
            parts = list(ex.map(build, graphs))
        # pack block-diagonally
        crow = [np.zeros(1, np.int64)]
        cols, vals, br, src, dst = [], [], [np.zeros(1, np.int64)], [], []
        nnz = 0
        edges = 0
        # where graph g's delta entries, tree edges and branch offsets start
        self.nnz_offsets = [0]
        self.edge_offsets = [0]
        self.branch_offsets = [0]
        if sum(s.csr_col.size for s in parts) >= 2 ** 31:
            raise RuntimeError("a batch holds fewer than 2^31 delta entries")
        for g, s in enumerate(parts):
            off = int(self.offsets[g])
            crow.append(s.csr_ptr[1:].astype(np.int64) + nnz)
            cols.append(s.csr_col.astype(np.int64) + off)
            vals.append(s.csr_val)
            br.append(s.branches[1:].astype(np.int64) + edges)
            src.append(s.src.astype(np.int64) + off)
            dst.append(s.dst.astype(np.int64) + off)
            nnz += s.csr_col.size
            edges += s.src.size
            self.nnz_offsets.append(nnz)
            self.edge_offsets.append(edges)
            self.branch_offsets.append(self.branch_offsets[-1] + s.branches.size - 1)
        self.nnz_a = int(sum(s.nnz_a for s in parts))
        crow = np.concatenate(crow).astype(np.int32)
        self.csr_ptr, self.csr_col = crow, np.concatenate(cols).astype(np.int32)
        self.csr_val = np.concatenate(vals).astype(np.float32)
        self.branches = np.concatenate(br).astype(np.int32)
        self.src = np.concatenate(src).astype(np.int32)
        self.dst = np.concatenate(dst).astype(np.int32)
        self.num_nodes = total
        self._plan = Plan(self.csr_ptr, self.csr_col, self.csr_val, total, total, self.branches, self.src, self.dst,
                          host=True)
        if op != "ax":
            # degrees through the product itself, as cbm4ad / cbm4dad do
            d = torch.zeros(total, 1, dtype=torch.float32, device="cuda")
            self._plan.matmul("ax", torch.ones(total, 1, dtype=torch.float32, device="cuda"), d)
            self.D = (d ** (-1 / 2)).view(-1)
            self._plan.set_multipliers(self.D)

    @property
    def plan(self):
        return self._plan

    def matmul(self, x, y):
        """y <- A_g x_g for every graph g; x, y: [total nodes, C], graph g in rows offsets[g]:offsets[g+1]."""
        self._plan.matmul(self.op, x, y)

    def split(self, t):
        """Per-graph views of a [total nodes, C] tensor."""
        return [t[int(self.offsets[g]): int(self.offsets[g + 1])] for g in range(len(self.sizes))]

    def graph_structure(self, g):
        """Graph g's own CBM structure, indices rebased to the graph: (row_ptr,
        col, val, branches, src, dst) as the reference's cbm_mkl_cpp.init and
        its products take them."""
        off = int(self.offsets[g])
        z0, z1 = self.nnz_offsets[g], self.nnz_offsets[g + 1]
        e0, e1 = self.edge_offsets[g], self.edge_offsets[g + 1]
        b0, b1 = self.branch_offsets[g], self.branch_offsets[g + 1]
        crow = self.csr_ptr[off:int(self.offsets[g + 1]) + 1].astype(np.int64) - z0
        return (crow.astype(np.int32), self.csr_col[z0:z1] - off, self.csr_val[z0:z1],
                self.branches[b0:b1 + 1] - e0, self.src[e0:e1] - off, self.dst[e0:e1] - off)

    def capture(self, x, y, warmup=2):
        """A CUDA graph that replays ``matmul(x, y)`` (x is read at replay time)."""
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            for _ in range(warmup):
                self.matmul(x, y)
        torch.cuda.current_stream().wait_stream(s)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            self.matmul(x, y)
        return graph
