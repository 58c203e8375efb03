"""``cbm4ad``: A D^-1/2 in CBM form, products Y = A D^-1/2 X (cbm/cbm4ad.py:5-42).

As in the reference, the degree d = A 1 is computed with the CBM product
itself (cbm/cbm4ad.py:11-16), D = d ** (-1/2) on the GPU (:19), and
``deltas`` carries the column-scaled values s * D[col] (:21-25).  The product
does not read those values: the kernel applies D[col] to each +-1 entry as it
gathers, which gives the same FP32 entry bit for bit.
"""
from __future__ import annotations

import torch

from .cbm4mm import cbm4mm
from .cbm_cusparse import cusparseCBM

__all__ = ["cbm4ad"]


class cbm4ad(cbm4mm):  # noqa: N801
    _op = "adx"
    _transpose_free_if_symmetric = False  # (A D^-1/2)^T = D^-1/2 A^T

    def __init__(self, edge_index, edge_values, alpha=0, cache_dir=None, cluster=None):
        super().__init__(edge_index, edge_values, alpha, cache_dir, cluster)
        num_rows = self.deltas.size()[0]
        d = torch.zeros(num_rows, 1, dtype=torch.float32, device="cuda")
        x = torch.ones(num_rows, 1, dtype=torch.float32, device="cuda")
        self._plan.matmul("ax", x, d)
        self.D = (d ** (-1 / 2)).view(-1)
        self._plan.set_multipliers(self.D)
        column_indices = self.deltas.col_indices()
        new_values = self.deltas.values() * self.D[column_indices]
        self.deltas = torch.sparse_csr_tensor(
            self.deltas.crow_indices().to(dtype=torch.int32),
            self.deltas.col_indices().to(dtype=torch.int32),
            new_values.to(dtype=torch.float32),
            self.deltas.shape).to(device="cuda")
        self.cusparse_extension = cusparseCBM._from_plan(self._plan, "adx", None, False)
