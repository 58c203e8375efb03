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

__all__ = ["init", "build", "build_cached", "save_structure", "load_structure", "Structure"]

# on-disk format: an .npz of every Structure array plus these scalars
_FORMAT = "cbm-structure-1"


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


def build(row, col, n_rows, alpha=0, n_threads=0, exhaustive=False, cluster=None):
    """Runs the constructor on COO indices (int32) and returns a Structure.
    cluster (int32 [n_rows], optional): restrict every row's parent to its own
    cluster (cbm_build_clustered)."""
    lib = _lib.load()
    row = _as_numpy_i32(row, "src_row_idx")
    col = _as_numpy_i32(col, "src_col_idx")
    if row.shape != col.shape or row.ndim != 1:
        raise RuntimeError("row and column index tensors must be 1-D and of equal length")
    n_rows = int(n_rows)
    h = C.c_void_p()
    flags = _lib.BUILD_EXHAUSTIVE if exhaustive else 0
    if cluster is None:
        rc = lib.cbm_build(row.ctypes.data, col.ctypes.data, row.size, n_rows, int(alpha), int(n_threads), flags,
                           C.byref(h))
    else:
        cl = np.ascontiguousarray(cluster, dtype=np.int32)
        if cl.shape != (n_rows,):
            raise RuntimeError(f"cluster must hold one id per row ({n_rows}), got {cl.shape}")
        rc = lib.cbm_build_clustered(row.ctypes.data, col.ctypes.data, row.size, n_rows, int(alpha),
                                     cl.ctypes.data, int(n_threads), flags, C.byref(h))
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


def save_structure(path, s, key=""):
    """Writes a Structure as an uncompressed .npz (atomically: a temporary file,
    then a rename).  ``key`` records what it was built from."""
    import os

    arrays = {name: getattr(s, name) for name, _, _ in _FIELDS}
    meta = np.array([s.n, s.n_candidates, s.tree_cost, s.nnz_a], dtype=np.int64)
    tmp = f"{path}.tmp{os.getpid()}"
    with open(tmp, "wb") as f:
        np.savez(f, _format=np.array(_FORMAT), _key=np.array(key), _meta=meta, **arrays)
    os.replace(tmp, path)


def load_structure(path, key=None):
    """Reads a Structure written by save_structure; None if the file is missing,
    of another format or (with ``key``) built from other input."""
    import os

    if not os.path.exists(path):
        return None
    with np.load(path) as d:
        if str(d["_format"]) != _FORMAT or (key is not None and str(d["_key"]) != key):
            return None
        n, cand, cost, nnz_a = (int(v) for v in d["_meta"])
        arrays = {name: d[name] for name, _, _ in _FIELDS}
    return Structure(n=n, n_candidates=cand, tree_cost=cost, nnz_a=nnz_a, **arrays)


def structure_key(row, col, n_rows, alpha, cluster=None):
    """SHA-1 of the edge list, the row count, alpha (and the cluster ids): names
    a cached structure."""
    import hashlib

    h = hashlib.sha1()
    parts = [_as_numpy_i32(row, "src_row_idx"), _as_numpy_i32(col, "src_col_idx")]
    if cluster is not None:
        parts.append(np.ascontiguousarray(cluster, dtype=np.int32))
    for a in parts:
        h.update(np.ascontiguousarray(a).view(np.uint8))
    h.update(f"|{int(n_rows)}|{int(alpha)}|{_FORMAT}".encode())
    return h.hexdigest()


def build_cached(row, col, n_rows, alpha=0, cache_dir=None, n_threads=0, cluster=None):
    """build() through an on-disk cache in ``cache_dir`` (none: plain build).
    Construction dominates set-up on large graphs (tens of seconds at millions
    of rows); the cache holds the six arrays of init plus the CSR form."""
    if not cache_dir:
        return build(row, col, n_rows, alpha, n_threads, cluster=cluster)
    import os

    os.makedirs(cache_dir, exist_ok=True)
    key = structure_key(row, col, n_rows, alpha, cluster)
    path = os.path.join(cache_dir, f"cbm-{key[:20]}.npz")
    s = load_structure(path, key)
    if s is None:
        s = build(row, col, n_rows, alpha, n_threads, cluster=cluster)
        save_structure(path, s, key)
    return s
