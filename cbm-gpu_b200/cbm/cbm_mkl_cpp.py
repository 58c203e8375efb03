"""CBM construction: the ``init`` operator of the reference's ``cbm_mkl_cpp`` module.

``init(row, col, values, n_rows, alpha)`` mirrors cbm_init_
(cbm/cbm_extensions.cpp:60-345, bound at :910): same argument meaning, the same
dtype checks (int32 indices, float32 values; a mismatch raises RuntimeError as
the reference's CHECK_DTYPE does, :14-16, :66-68) and the same six CPU tensors
in the same order:

    [delta_row int32[Z], delta_col int32[Z], delta_val float32[Z] (+-1),
     mca_branches int32[B+1], mca_src int32[E] (parents), mca_dst int32[E]]

It runs the native OpenMP constructor in libcbm_b200.so (no MKL, no arbok).
The reference's CPU products (s_spmm_update_csr_int32 and friends) are not part
of this module: the products run on the GPU (cbm.cbm_cusparse / cbm.cbm4*).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib

__all__ = ["init", "build", "Structure"]


@dataclass
class Structure:
    """Everything the constructor produces (numpy, host)."""

    n: int
    delta_row: np.ndarray
    delta_col: np.ndarray
    delta_val: np.ndarray
    branches: np.ndarray
    src: np.ndarray
    dst: np.ndarray
    parent: np.ndarray     # int32 [N], N marks the virtual root
    csr_ptr: np.ndarray    # delta matrix as CSR
    csr_col: np.ndarray
    csr_val: np.ndarray
    n_candidates: int
    tree_cost: int
    nnz_a: int


_FIELDS = [
    ("delta_row", _lib.S_DELTA_ROW, np.int32),
    ("delta_col", _lib.S_DELTA_COL, np.int32),
    ("delta_val", _lib.S_DELTA_VAL, np.float32),
    ("branches", _lib.S_BRANCHES, np.int32),
    ("src", _lib.S_SRC, np.int32),
    ("dst", _lib.S_DST, np.int32),
    ("parent", _lib.S_PARENT, np.int32),
    ("csr_ptr", _lib.S_CSR_PTR, np.int32),
    ("csr_col", _lib.S_CSR_COL, np.int32),
    ("csr_val", _lib.S_CSR_VAL, np.float32),
]


def _as_numpy_i32(t, name):
    if isinstance(t, torch.Tensor):
        if t.dtype != torch.int32:
            raise RuntimeError(f'"{name}" is not a tensor of type "torch::kInt32"')
        return np.ascontiguousarray(t.detach().cpu().numpy())
    a = np.asarray(t)
    if a.dtype != np.int32:
        raise RuntimeError(f'"{name}" is not a tensor of type "torch::kInt32"')
    return np.ascontiguousarray(a)


def build(row, col, n_rows, alpha=0, n_threads=0, exhaustive=False):
    """Runs the constructor on COO indices (int32) and returns a Structure."""
    lib = _lib.load()
    row = _as_numpy_i32(row, "src_row_idx")
    col = _as_numpy_i32(col, "src_col_idx")
    if row.shape != col.shape or row.ndim != 1:
        raise RuntimeError("row and column index tensors must be 1-D and of equal length")
    n_rows = int(n_rows)
    h = C.c_void_p()
    rc = lib.cbm_build(row.ctypes.data, col.ctypes.data, row.size, n_rows, int(alpha), int(n_threads),
                       _lib.BUILD_EXHAUSTIVE if exhaustive else 0, C.byref(h))
    _lib.check(rc, "cbm_build")
    try:
        out = {}
        for name, which, dt in _FIELDS:
            n = lib.cbm_structure_len(h, which)
            a = np.empty(n, dtype=dt)
            if n:
                _lib.check(lib.cbm_structure_copy(h, which, a.ctypes.data), "cbm_structure_copy")
            out[name] = a
        return Structure(
            n=n_rows,
            n_candidates=int(lib.cbm_structure_len(h, _lib.S_N_CANDIDATES)),
            tree_cost=int(lib.cbm_structure_len(h, _lib.S_TREE_COST)),
            nnz_a=int(lib.cbm_structure_len(h, _lib.S_NNZ_A)),
            **out,
        )
    finally:
        lib.cbm_structure_free(h)


def init(src_row_idx, src_col_idx, src_values, src_n_rows, alpha):
    """The reference's ``cbm_mkl_cpp.init`` (cbm/cbm_extensions.cpp:60-345)."""
    if isinstance(src_values, torch.Tensor):
        if src_values.dtype != torch.float32:
            raise RuntimeError('"src_values" is not a tensor of type "torch::kFloat32"')
    elif np.asarray(src_values).dtype != np.float32:
        raise RuntimeError('"src_values" is not a tensor of type "torch::kFloat32"')
    s = build(src_row_idx, src_col_idx, int(src_n_rows), int(alpha))
    return [torch.from_numpy(getattr(s, f)) for f in
            ("delta_row", "delta_col", "delta_val", "branches", "src", "dst")]
