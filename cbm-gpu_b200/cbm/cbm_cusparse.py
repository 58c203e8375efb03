"""Drop-in for the reference's ``cbm_cusparse`` extension module (cbm/cbm.cu:302-310).

``cusparseCBM(deltas, mca_branches, mca_src_node_idx, mca_dst_node_idx,
multipliers)`` takes the same CUDA tensors as the reference class
(cbm/cbm.cu:95-142); ``matmul_AX_ADX(rhs, res)`` and
``matmul_DAX_DADX(rhs, res)`` compute the same products (cbm/cbm.cu:150-268)
and return 0.  No cuSPARSE is involved: both run the fused sm_100a kernel of
libcbm_b200.so on the current stream, with no per-call allocation.

Differences, all in the direction of checking more: dtypes, shapes, devices
and the tree structure are validated and raise RuntimeError (the reference
prints and continues, cbm/cbm.cu:7-23); matmul_DAX_DADX without multipliers
raises instead of dereferencing an unset pointer (cbm/cbm.cu:139-140, :261).
"""
from __future__ import annotations

import torch

from .plan import Plan

__all__ = ["cusparseCBM"]


def _check_cuda(t):
    if not (isinstance(t, torch.Tensor) and t.is_cuda):
        raise RuntimeError("tensor is not a CUDA tensor")


class cusparseCBM:  # noqa: N801 (the reference's class name)
    """CBM product operator over a delta matrix and a compression tree."""

    def __init__(self, deltas, mca_branches, mca_src_node_idx, mca_dst_node_idx, multipliers):
        _check_cuda(deltas)
        _check_cuda(mca_branches)
        _check_cuda(mca_src_node_idx)
        _check_cuda(mca_dst_node_idx)
        if multipliers.numel():
            _check_cuda(multipliers)
        if deltas.layout != torch.sparse_csr:
            raise RuntimeError("deltas must be a torch.sparse_csr tensor")
        n_rows, n_cols = int(deltas.size(0)), int(deltas.size(1))
        self._plan = Plan(deltas.crow_indices(), deltas.col_indices(), deltas.values(), n_rows, n_cols,
                          mca_branches, mca_src_node_idx, mca_dst_node_idx,
                          multipliers if multipliers.numel() else None, host=False)
        self._has_mult = bool(multipliers.numel())
        self._ops = ("values_add", "values_ratio")

    @classmethod
    def _from_plan(cls, plan, op_add, op_ratio, has_mult):
        obj = cls.__new__(cls)
        obj._plan = plan
        obj._ops = (op_add, op_ratio)
        obj._has_mult = has_mult
        return obj

    @property
    def plan(self):
        return self._plan

    def matmul_AX_ADX(self, rhs, res):  # noqa: N802
        _check_cuda(rhs)
        _check_cuda(res)
        self._plan.matmul(self._ops[0], rhs, res)
        return 0

    def matmul_DAX_DADX(self, rhs, res):  # noqa: N802
        _check_cuda(rhs)
        _check_cuda(res)
        if not self._has_mult or self._ops[1] is None:
            raise RuntimeError("matmul_DAX_DADX needs multipliers")
        self._plan.matmul(self._ops[1], rhs, res)
        return 0
