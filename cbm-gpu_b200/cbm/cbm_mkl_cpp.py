"""The reference's ``cbm_mkl_cpp`` module (cbm/cbm_extensions.cpp:909-919):
the constructor ``init`` and the eight products, with the reference's names,
argument lists and in-place ``dst``.

``init(row, col, values, n_rows, alpha)`` mirrors cbm_init_
(cbm/cbm_extensions.cpp:60-345, bound at :910): same argument meaning, the same
dtype checks (int32 indices, float32 values; a mismatch raises RuntimeError as
the reference's CHECK_DTYPE does, :14-16, :66-68) and the same six CPU tensors
in the same order:

    [delta_row int32[Z], delta_col int32[Z], delta_val float32[Z] (+-1),
     mca_branches int32[B+1], mca_src int32[E] (parents), mca_dst int32[E]]

It runs the native OpenMP constructor in libcbm_b200.so (no MKL, no arbok).

The products (``s_spmm_update_csr_int32`` and the seven others, :351-907) run
on the GPU through the library's stateless ``cbm_s_*`` entry points
(include/cbm_b200.h), straight from the arguments' CSR arrays and tree edges:

* CUDA tensors (all on one device): the call is queued on the current stream
  and returns at once, like any CUDA operator; device-side errors (an index
  out of range, a node with two parents, a child edge listed before its
  parent's) are recorded and raised by ``check_device()``.
* CPU tensors (the reference's own convention): the operands are copied to the
  current CUDA device, the product runs there and ``dst`` is filled in place
  on return; device-side errors raise at once.

Rounding follows the reference's CPU path: each row sums its entries in order
with one FMA each (MKL may order them differently, so results agree within
rounding, not bit for bit); the fused update is fma(Y[u], m[v] / m[u], Y[v]);
the GIN term is fma(1 + eps, X, Y).  ``s_spmm_csr_t_int32`` adds with atomics,
in no fixed order.  There is no CPU fallback: without a CUDA device the
products raise RuntimeError.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib

__all__ = ["init", "build", "build_cached", "save_structure", "load_structure", "Structure",
           "s_spmm_update_csr_int32", "s_spmm_fused_update_csr_int32", "s_spmm_add_csr_int32",
           "s_spmm_update_add_csr_int32", "s_spmm_csr_int32", "s_spmm_csr_t_int32", "s_update_csr_int32",
           "s_fused_update_csr_int32", "device_status", "check_device"]

# on-disk format: an .npz of every Structure array plus these scalars
_FORMAT = "cbm-structure-2"


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
    symmetric: bool = False  # A == A^T


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
            symmetric=bool(lib.cbm_structure_len(h, _lib.S_SYMMETRIC)),
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
    meta = np.array([s.n, s.n_candidates, s.tree_cost, s.nnz_a, int(s.symmetric)], dtype=np.int64)
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
        n, cand, cost, nnz_a, sym = (int(v) for v in d["_meta"])
        arrays = {name: d[name] for name, _, _ in _FIELDS}
    return Structure(n=n, n_candidates=cand, tree_cost=cost, nnz_a=nnz_a, symmetric=bool(sym), **arrays)


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


# ---- the reference's CPU products, on the GPU ------------------------------------

_WORKSPACE = {}  # device index -> zero-filled uint8 tensor (status word + per-node stamps)


def _workspace(device, rows):
    """The device's workspace, grown to ``rows`` nodes (its status word carried over)."""
    lib = _lib.load()
    need = max(int(lib.cbm_direct_workspace_bytes(int(rows))), 256)
    ws = _WORKSPACE.get(device.index)
    if ws is None or ws.numel() < need:
        grown = torch.zeros(max(need, 2 * ws.numel() if ws is not None else 0), dtype=torch.uint8, device=device)
        if ws is not None:
            grown[:256].copy_(ws[:256])
        _WORKSPACE[device.index] = ws = grown
    return ws


def device_status(device=None):
    """Synchronises the current stream of ``device`` and returns (status, info):
    the first device-side error the products recorded since the last query
    (status 0: none), then clears it."""
    device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    ws = _WORKSPACE.get(device.index)
    if ws is None:
        return _lib.OK, 0
    st = C.c_int32(0)
    info = C.c_int64(0)
    with torch.cuda.device(device):
        _lib.check(_lib.load().cbm_direct_status(ws.data_ptr(), C.c_void_p(torch.cuda.current_stream().cuda_stream),
                                                 C.byref(st), C.byref(info)), "cbm_direct_status")
    return int(st.value), int(info.value)


def check_device(device=None):
    """Raises CbmError if a product on ``device`` recorded a device-side error."""
    st, info = device_status(device)
    if st != _lib.OK:
        raise _lib.CbmError(st, f"device-side error in a cbm_mkl_cpp product (at {info})")


def _check_dtype(t, name, dt):
    if not isinstance(t, torch.Tensor) or t.dtype != dt:
        tn = {torch.float32: "torch::kFloat32", torch.int32: "torch::kInt32"}[dt]
        raise RuntimeError(f'"{name}" is not a tensor of type "{tn}"')


def _run(entry, named, make_args):
    """Checks dtypes (in the reference's order), then shapes (``make_args()``
    checks them and returns ``build_args``) and devices, moves CPU operands to
    the GPU and back, and calls ``entry`` with the device pointers
    ``build_args(ptr, stream, ws)`` lays out."""
    lib = _lib.load()
    for name, t, dt in named:
        _check_dtype(t, name, dt)
    build_args = make_args()
    tensors = {name: t for name, t, _ in named}
    on_cuda = {t.is_cuda for t in tensors.values()}
    if len(on_cuda) != 1:
        raise RuntimeError("all tensors must be on the same device (all CUDA or all CPU)")
    host = not on_cuda.pop()
    if not torch.cuda.is_available():
        raise RuntimeError("cbm_mkl_cpp products run on a CUDA device; none is available")
    if host:
        device = torch.device("cuda", torch.cuda.current_device())
        dev = {name: t.contiguous().to(device, non_blocking=False) for name, t in tensors.items()}
    else:
        devices = {t.device for t in tensors.values()}
        if len(devices) != 1:
            raise RuntimeError(f"tensors are on several devices: {sorted(str(d) for d in devices)}")
        device = devices.pop()
        for name, t in tensors.items():
            if not t.is_contiguous():
                raise RuntimeError(f'"{name}" must be contiguous')
        dev = tensors
    with torch.cuda.device(device):
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        out = dev["dst"]
        ws = _workspace(device, out.shape[0])

        def ptr(name):
            t = dev[name]
            return t.data_ptr() if t.numel() else None

        rc = getattr(lib, entry)(*build_args(ptr, stream, ws))
        _lib.check(rc, entry)
        if host:
            tensors["dst"].copy_(out.cpu())
            check_device(device)


def _csr_sizes(rp_b, rp_e, col, val, rows):
    if rp_b.dim() != 1 or rp_e.dim() != 1 or rp_b.numel() != rows or rp_e.numel() != rows:
        raise RuntimeError(f"row pointers must hold one entry per row ({rows}): got {rp_b.numel()}, {rp_e.numel()}")
    if col.dim() != 1 or val.dim() != 1 or col.numel() != val.numel():
        raise RuntimeError("lhs_col_idx and lhs_values must be 1-D and of equal length")
    return col.numel()


def _dense(t, name, rows=None, cols=None):
    if t.dim() != 2 or (rows is not None and t.shape[0] != rows) or (cols is not None and t.shape[1] != cols):
        raise RuntimeError(f'"{name}": expected a [{rows if rows is not None else "N"}, '
                           f'{cols if cols is not None else "C"}] matrix, got {list(t.shape)}')


def _tree_sizes(branches, src, dst_idx):
    if branches.dim() != 1 or src.dim() != 1 or dst_idx.dim() != 1 or src.numel() != dst_idx.numel():
        raise RuntimeError("mca_row_idx and mca_col_idx must be 1-D and of equal length")
    return branches.numel(), src.numel()


_I32, _F32 = torch.int32, torch.float32


def _spmm_named(lhs_row_ptr_b, lhs_row_ptr_e, lhs_col_idx, lhs_values, rhs, dst, tree=(), mult=None):
    named = [("rhs", rhs, _F32), ("dst", dst, _F32)]
    if tree:
        named += [("mca_branches", tree[0], _I32), ("mca_row_idx", tree[1], _I32), ("mca_col_idx", tree[2], _I32)]
    named += [("lhs_row_ptr_b", lhs_row_ptr_b, _I32), ("lhs_row_ptr_e", lhs_row_ptr_e, _I32),
              ("lhs_col_idx", lhs_col_idx, _I32), ("lhs_values", lhs_values, _F32)]
    if mult is not None:
        named.append(("multiplier", mult, _F32))
    return named


def s_spmm_update_csr_int32(lhs_row_ptr_b, lhs_row_ptr_e, lhs_col_idx, lhs_values, rhs, mca_branches, mca_row_idx,
                            mca_col_idx, dst):
    """dst = Delta rhs, then dst[child] += dst[parent] along the tree
    (cbm/cbm_extensions.cpp:351-444)."""
    named = _spmm_named(lhs_row_ptr_b, lhs_row_ptr_e, lhs_col_idx, lhs_values, rhs, dst,
                        (mca_branches, mca_row_idx, mca_col_idx))
    _run("cbm_s_spmm_update_csr_int32", named, lambda: _spmm_tree_args(named, rhs, dst, False, None))


def s_spmm_fused_update_csr_int32(lhs_row_ptr_b, lhs_row_ptr_e, lhs_col_idx, lhs_values, rhs, mca_branches,
                                  mca_row_idx, mca_col_idx, multiplier, dst):
    """dst = Delta rhs, then dst[child] = fma(dst[parent], m[child] / m[parent],
    dst[child]) along the tree (cbm/cbm_extensions.cpp:593-698)."""
    named = _spmm_named(lhs_row_ptr_b, lhs_row_ptr_e, lhs_col_idx, lhs_values, rhs, dst,
                        (mca_branches, mca_row_idx, mca_col_idx), multiplier)
    _run("cbm_s_spmm_fused_update_csr_int32", named, lambda: _spmm_tree_args(named, rhs, dst, True, None))


def s_spmm_update_add_csr_int32(lhs_row_ptr_b, lhs_row_ptr_e, lhs_col_idx, lhs_values, rhs, epsilon, mca_branches,
                                mca_row_idx, mca_col_idx, dst):
    """dst = Delta rhs, the update, then dst += (1 + epsilon) rhs: the CBM GIN
    aggregation (cbm/cbm_extensions.cpp:494-591)."""
    named = _spmm_named(lhs_row_ptr_b, lhs_row_ptr_e, lhs_col_idx, lhs_values, rhs, dst,
                        (mca_branches, mca_row_idx, mca_col_idx))
    _run("cbm_s_spmm_update_add_csr_int32", named,
         lambda: _spmm_tree_args(named, rhs, dst, False, float(epsilon)))


def _spmm_tree_args(named, rhs, dst, fused, epsilon):
    t = {name: v for name, v, _ in named}
    _dense(dst, "dst")
    _dense(rhs, "rhs", cols=dst.shape[1])
    n_rows = int(dst.shape[0])
    nnz = _csr_sizes(t["lhs_row_ptr_b"], t["lhs_row_ptr_e"], t["lhs_col_idx"], t["lhs_values"], n_rows)
    if epsilon is not None and rhs.shape[0] != n_rows:
        raise RuntimeError(f"the (1 + epsilon) rhs term needs a square matrix: rhs has {rhs.shape[0]} rows, "
                           f"dst {n_rows}")
    n_br, n_edges = _tree_sizes(t["mca_branches"], t["mca_row_idx"], t["mca_col_idx"])
    if fused and (t["multiplier"].dim() != 1 or t["multiplier"].numel() != n_rows):
        raise RuntimeError(f'"multiplier" must hold one entry per row ({n_rows})')

    def build(ptr, stream, ws):
        head = [ptr("lhs_row_ptr_b"), ptr("lhs_row_ptr_e"), ptr("lhs_col_idx"), ptr("lhs_values"), n_rows,
                int(rhs.shape[0]), nnz, ptr("rhs"), int(rhs.shape[1])]
        if epsilon is not None:
            head.append(C.c_float(epsilon))
        tree = [ptr("mca_branches"), n_br, ptr("mca_row_idx"), ptr("mca_col_idx"), n_edges]
        if fused:
            tree.append(ptr("multiplier"))
        return head + tree + [ptr("dst"), ws.data_ptr(), ws.numel(), stream]

    return build


def _spmm_plain(entry, lhs_row_ptr_b, lhs_row_ptr_e, lhs_col_idx, lhs_values, rhs, dst, transpose=False,
                epsilon=None):
    named = _spmm_named(lhs_row_ptr_b, lhs_row_ptr_e, lhs_col_idx, lhs_values, rhs, dst)
    _run(entry, named, lambda: _plain_args(lhs_row_ptr_b, lhs_row_ptr_e, lhs_col_idx, lhs_values, rhs, dst, transpose,
                                           epsilon))


def _plain_args(lhs_row_ptr_b, lhs_row_ptr_e, lhs_col_idx, lhs_values, rhs, dst, transpose, epsilon):
    _dense(dst, "dst")
    _dense(rhs, "rhs", cols=dst.shape[1])
    if transpose:
        # A [rows of rhs, rows of dst]: dst = A^T rhs
        n_rows, n_cols = int(rhs.shape[0]), int(dst.shape[0])
    else:
        n_rows, n_cols = int(dst.shape[0]), int(rhs.shape[0])
    if epsilon is not None and n_rows != n_cols:
        raise RuntimeError(f"the (1 + epsilon) rhs term needs a square matrix: rhs has {n_cols} rows, dst {n_rows}")
    nnz = _csr_sizes(lhs_row_ptr_b, lhs_row_ptr_e, lhs_col_idx, lhs_values, n_rows)

    def build(ptr, stream, ws):
        args = [ptr("lhs_row_ptr_b"), ptr("lhs_row_ptr_e"), ptr("lhs_col_idx"), ptr("lhs_values"), n_rows, n_cols,
                nnz, ptr("rhs"), int(rhs.shape[1])]
        if epsilon is not None:
            args.append(C.c_float(epsilon))
        return args + [ptr("dst"), ws.data_ptr(), ws.numel(), stream]

    return build


def s_spmm_csr_int32(lhs_row_ptr_b, lhs_row_ptr_e, lhs_col_idx, lhs_values, rhs, dst):
    """dst = A rhs (cbm/cbm_extensions.cpp:700-740)."""
    _spmm_plain("cbm_s_spmm_csr_int32", lhs_row_ptr_b, lhs_row_ptr_e, lhs_col_idx, lhs_values, rhs, dst)


def s_spmm_csr_t_int32(lhs_row_ptr_b, lhs_row_ptr_e, lhs_col_idx, lhs_values, rhs, dst):
    """dst = A^T rhs, A with one row per row of rhs (cbm/cbm_extensions.cpp:742-782,
    where A is square)."""
    _spmm_plain("cbm_s_spmm_csr_t_int32", lhs_row_ptr_b, lhs_row_ptr_e, lhs_col_idx, lhs_values, rhs, dst,
                transpose=True)


def s_spmm_add_csr_int32(lhs_row_ptr_b, lhs_row_ptr_e, lhs_col_idx, lhs_values, rhs, epsilon, dst):
    """dst = A rhs + (1 + epsilon) rhs: the GIN aggregation over CSR
    (cbm/cbm_extensions.cpp:446-492)."""
    _spmm_plain("cbm_s_spmm_add_csr_int32", lhs_row_ptr_b, lhs_row_ptr_e, lhs_col_idx, lhs_values, rhs, dst,
                epsilon=float(epsilon))


def _update(entry, mca_branches, mca_row_idx, mca_col_idx, dst, multiplier=None):
    named = [("dst", dst, _F32), ("mca_branches", mca_branches, _I32), ("mca_row_idx", mca_row_idx, _I32),
             ("mca_col_idx", mca_col_idx, _I32)]
    if multiplier is not None:
        named.append(("multiplier", multiplier, _F32))
    _run(entry, named, lambda: _update_args(mca_branches, mca_row_idx, mca_col_idx, dst, multiplier))


def _update_args(mca_branches, mca_row_idx, mca_col_idx, dst, multiplier):
    _dense(dst, "dst")
    n_br, n_edges = _tree_sizes(mca_branches, mca_row_idx, mca_col_idx)
    if multiplier is not None and (multiplier.dim() != 1 or multiplier.numel() != dst.shape[0]):
        raise RuntimeError(f'"multiplier" must hold one entry per row ({dst.shape[0]})')

    def build(ptr, stream, ws):
        args = [ptr("mca_branches"), n_br, ptr("mca_row_idx"), ptr("mca_col_idx"), n_edges]
        if multiplier is not None:
            args.append(ptr("multiplier"))
        return args + [ptr("dst"), int(dst.shape[0]), int(dst.shape[1]), ws.data_ptr(), ws.numel(), stream]

    return build


def s_update_csr_int32(mca_branches, mca_row_idx, mca_col_idx, dst):
    """dst[child] += dst[parent] along the tree, in place (cbm/cbm_extensions.cpp:784-838)."""
    _update("cbm_s_update_csr_int32", mca_branches, mca_row_idx, mca_col_idx, dst)


def s_fused_update_csr_int32(mca_branches, mca_row_idx, mca_col_idx, multiplier, dst):
    """dst[child] = fma(dst[parent], m[child] / m[parent], dst[child]) along the
    tree, in place (cbm/cbm_extensions.cpp:841-907)."""
    _update("cbm_s_fused_update_csr_int32", mca_branches, mca_row_idx, mca_col_idx, dst, multiplier)
