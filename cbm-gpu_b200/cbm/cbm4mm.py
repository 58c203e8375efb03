"""``cbm4mm``: A stored in CBM form, products Y = A X (cbm/cbm4mm.py:7-54).

Same constructor arguments (edge_index int32 [2, nnz], edge_values float32
[nnz], alpha) and attributes (deltas, num_nodes, mca_offset, mca_src_idx,
mca_dst_idx, cusparse_extension) as the reference class.  ``matmul(x, y)``
writes A x into the preallocated y, on the current stream.

Beyond the reference: x may be bfloat16 (y float32 or bfloat16, FP32
accumulation), ``forward(x)`` is differentiable through torch.autograd
(the adjoint runs in CBM form), and ``adjoint(g, dx)`` computes A^T g.
"""
from __future__ import annotations

import torch

from . import cbm_mkl_cpp as cbm_mkl
from .cbm_cusparse import cusparseCBM
from .plan import Plan

__all__ = ["cbm4mm"]


class cbm4mm:  # noqa: N801 (the reference's class name)
    _op = "ax"
    # the operator equals its transpose when A does (A, D^-1/2 A D^-1/2; not A D^-1/2)
    _transpose_free_if_symmetric = True

    def __init__(self, edge_index, edge_values, alpha=0, cache_dir=None, cluster=None):
        """Additions to the reference's arguments: cache_dir reuses the
        constructed structure from an on-disk cache keyed by the edge list and
        alpha (cbm_mkl_cpp.build_cached); cluster (int32 per row, e.g.
        cbm.cluster.cluster_ids of LSH clusters) restricts every row's parent
        to its own cluster: the reference's per-cluster CBMs as one operator."""
        if edge_index.numel() == 0:
            raise RuntimeError("edge_index is empty")
        num_rows = int(max(edge_index[0].max(), edge_index[1].max())) + 1
        if isinstance(edge_values, torch.Tensor) and edge_values.dtype != torch.float32:
            raise RuntimeError('"src_values" is not a tensor of type "torch::kFloat32"')
        s = cbm_mkl.build_cached(edge_index[0], edge_index[1], num_rows, alpha, cache_dir, cluster=cluster)
        self.structure_stats = {"nnz_a": s.nnz_a, "nnz_delta": int(s.csr_col.size), "edges": int(s.src.size),
                                "branches": int(s.branches.size) - 1, "candidates": s.n_candidates}
        self.deltas = torch.sparse_csr_tensor(
            torch.from_numpy(s.csr_ptr), torch.from_numpy(s.csr_col), torch.from_numpy(s.csr_val),
            (num_rows, num_rows)).to(device="cuda")
        self.num_nodes = num_rows
        self.mca_offset = torch.from_numpy(s.branches).to(dtype=torch.int32, device="cuda")
        self.mca_src_idx = torch.from_numpy(s.src).to(dtype=torch.int32, device="cuda")
        self.mca_dst_idx = torch.from_numpy(s.dst).to(dtype=torch.int32, device="cuda")
        self.parent = s.parent  # host int32 [N], N = virtual root
        self.symmetric = bool(s.symmetric)  # A == A^T (found by the constructor)
        self._plan = Plan(s.csr_ptr, s.csr_col, s.csr_val, num_rows, num_rows, s.branches, s.src, s.dst,
                          host=True)
        self.cusparse_extension = cusparseCBM._from_plan(self._plan, "ax", None, False)

    @property
    def plan(self):
        return self._plan

    def matmul(self, x, y):
        self._plan.matmul(self._op, x, y)

    def matmul_add(self, x, y, epsilon=0.0):
        """y <- A x + (1 + epsilon) x: the GIN aggregation the reference computes
        on the CPU only (s_spmm_update_add_csr_int32,
        cbm/cbm_extensions.cpp:498-591), with the binary A of this matrix."""
        self._plan.matmul_gin(x, y, epsilon)

    def matmul_host(self, x, y, slab_cols=64, overlap_calls=False):
        """y <- (this operator) x for host tensors x and y (pinned for full-speed
        copies), the copies overlapped with the product slab by slab.  Queued on
        the current stream: synchronise it before reading y.  overlap_calls:
        back-to-back calls also overlap one call's copy-out with the next
        call's copy-in (x must be complete in host memory at the call), and the
        current stream waits only for the products: call host_wait() before
        synchronising to read y."""
        self._plan.matmul_host(self._op, x, y, slab_cols, overlap_calls)

    def host_wait(self):
        """The current stream waits for every copy-out of matmul_host calls so
        far (after calls with overlap_calls)."""
        self._plan.host_wait()

    @property
    def self_adjoint(self):
        """True when this operator equals its transpose (A symmetric, and the
        operator A or D^-1/2 A D^-1/2): then A^T g = A g."""
        return self.symmetric and self._transpose_free_if_symmetric

    def adjoint(self, g, dx):
        """dx <- (this operator)^T g, by the adjoint kernels (reverse tree
        propagation, then the transposed-delta gather)."""
        self._plan.adjoint(self._op, g, dx)

    def forward(self, x, out_dtype=None):
        """Differentiable y = (this operator) x; y has x's dtype unless out_dtype is given."""
        from .autograd import cbm_apply
        return cbm_apply(self, x, out_dtype)

    __call__ = forward
