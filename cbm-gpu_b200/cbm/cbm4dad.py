"""``cbm4dad``: D^-1/2 A D^-1/2 in CBM form (cbm/cbm4dad.py:5-54).

Degree and D as in cbm4ad (cbm/cbm4dad.py:11-19).  ``deltas`` carries the
values (s * D[col]) * D[row] that the reference prepares (:21-34; its
``missing_nodes`` set holds every row, so every row is scaled), computed here
without the per-row Python loop.  The product uses the reference's propagation
rule Y[v] += Y[u] * D[v] / D[u] (cbm/cbm.cu:88) and forms each entry as
(s * D[col]) * D[row] on the fly, as the reference's prepared values are.
"""
from __future__ import annotations

import torch

from .cbm4mm import cbm4mm
from .cbm_cusparse import cusparseCBM

__all__ = ["cbm4dad"]


class cbm4dad(cbm4mm):  # noqa: N801
    _op = "dadx"

    def __init__(self, edge_index, edge_values, alpha=0, cache_dir=None, cluster=None):
        super().__init__(edge_index, edge_values, alpha, cache_dir, cluster)
        num_rows = self.deltas.size()[0]
        d = torch.zeros(num_rows, 1, dtype=torch.float32, device="cuda")
        x = torch.ones(num_rows, 1, dtype=torch.float32, device="cuda")
        self._plan.matmul("ax", x, d)
        self.D = (d ** (-1 / 2)).view(-1)
        self._plan.set_multipliers(self.D)
        crow = self.deltas.crow_indices()
        column_indices = self.deltas.col_indices()
        new_values = self.deltas.values() * self.D[column_indices]
        row_of_entry = torch.repeat_interleave(torch.arange(num_rows, device="cuda"), torch.diff(crow))
        new_values = new_values * self.D[row_of_entry]
        self.deltas = torch.sparse_csr_tensor(
            crow.to(dtype=torch.int32), column_indices.to(dtype=torch.int32),
            new_values.to(dtype=torch.float32), self.deltas.shape).to(device="cuda")
        self.cusparse_extension = cusparseCBM._from_plan(self._plan, "dad_add", "dadx", True)
