"""Python face of the CPU oracle (cbm_oracle.c) -- TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
checker / CPU baseline; the product (cbm-gpu_b200/) never imports it.
Each function names the reference code it restates.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None

vp, i64, i32 = C.c_void_p, C.c_int64, C.c_int32


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.oracle_candidates.restype = i64
        L.oracle_candidates.argtypes = [i64, vp, vp, i64, i64, vp, vp, vp]
        L.oracle_arb_cost.restype = i64
        L.oracle_arb_cost.argtypes = [i64, i64, i64, vp, vp, vp]
        L.oracle_emit.restype = C.c_int
        L.oracle_emit.argtypes = [i64, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        for name in ("oracle_spmm_update", "oracle_spmm_update_omp"):
            f = getattr(L, name)
            f.restype = None
            f.argtypes = [i64, i64, vp, vp, vp, vp, i64, vp, vp, vp, vp]
        L.oracle_spmm_fused_update.restype = None
        L.oracle_spmm_fused_update.argtypes = [i64, i64, vp, vp, vp, vp, i64, vp, vp, vp, vp, i32, vp]
        L.oracle_spmm_fused_update_omp.restype = None
        L.oracle_spmm_fused_update_omp.argtypes = [i64, i64, vp, vp, vp, vp, i64, vp, vp, vp, vp, vp]
        L.oracle_csr_spmm_f64.restype = None
        L.oracle_csr_spmm_f64.argtypes = [i64, i64, vp, vp, i64, vp, vp, vp, i32, vp]
        L.oracle_threads.restype = C.c_int
        _lib = L
    return _lib


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def csr_from_edges(edge_index, n):
    """Binary CSR (sorted, unique columns) of edge_index; int64 row pointers."""
    r = np.asarray(edge_index[0], dtype=np.int64)
    c = np.asarray(edge_index[1], dtype=np.int64)
    key = np.unique(r * n + c)
    rows = key // n
    cols = (key % n).astype(np.int32)
    ptr = np.zeros(n + 1, dtype=np.int64)
    ptr[1:] = np.cumsum(np.bincount(rows, minlength=n))
    return ptr, cols


def candidates(ptr, idx, alpha):
    """The reference's candidate list G (cbm/cbm_extensions.cpp:123-151), brute force."""
    n = ptr.size - 1
    ptr = _c(ptr, np.int64)
    idx = _c(idx, np.int32)
    cap = n + 2 * n * n
    cap = min(cap, 50_000_000)
    f = np.empty(cap, np.int32)
    t = np.empty(cap, np.int32)
    w = np.empty(cap, np.int64)
    m = lib().oracle_candidates(n, ptr.ctypes.data, idx.ctypes.data, int(alpha), cap, f.ctypes.data,
                                t.ctypes.data, w.ctypes.data)
    if m < 0:
        raise RuntimeError("candidate list too large for the oracle")
    return f[:m].copy(), t[:m].copy(), w[:m].copy()


def arborescence_cost(n_nodes, root, f, t, w):
    """Optimum arborescence cost (textbook Chu-Liu/Edmonds)."""
    f, t, w = _c(f, np.int32), _c(t, np.int32), _c(w, np.int64)
    return int(lib().oracle_arb_cost(n_nodes, root, f.size, f.ctypes.data, t.ctypes.data, w.ctypes.data))


def emit(ptr, idx, f, in_edge):
    """BFS emission (cbm/cbm_extensions.cpp:191-299) for given tree in-edges.

    Returns the six arrays of cbm_init_ (delta_row, delta_col, delta_val,
    branches, src, dst)."""
    n = ptr.size - 1
    ptr, idx, f, in_edge = _c(ptr, np.int64), _c(idx, np.int32), _c(f, np.int32), _c(in_edge, np.int32)
    cap = 2 * idx.size + 1
    dr = np.empty(cap, np.int32)
    dc = np.empty(cap, np.int32)
    dv = np.empty(cap, np.float32)
    br = np.empty(n + 2, np.int32)
    s = np.empty(max(n, 1), np.int32)
    d = np.empty(max(n, 1), np.int32)
    cnt = np.zeros(3, np.int64)
    lib().oracle_emit(n, ptr.ctypes.data, idx.ctypes.data, f.ctypes.data, in_edge.ctypes.data, dr.ctypes.data,
                      dc.ctypes.data, dv.ctypes.data, br.ctypes.data, s.ctypes.data, d.ctypes.data, cnt.ctypes.data)
    z, e, b1 = (int(v) for v in cnt)
    return dr[:z].copy(), dc[:z].copy(), dv[:z].copy(), br[:b1].copy(), s[:e].copy(), d[:e].copy()


def reference_structure(edge_index, n, alpha, parent):
    """Candidate list + emission for a given parent choice (parent[v] == n: root).

    Returns (six arrays, in_edge) or raises if some parent edge is not a
    candidate of the reference's rules."""
    ptr, idx = csr_from_edges(edge_index, n)
    f, t, w = candidates(ptr, idx, alpha)
    lookup = {(int(a), int(b)): i for i, (a, b) in enumerate(zip(f, t))}
    in_edge = np.empty(n, np.int32)
    for v in range(n):
        key = (int(parent[v]), v)
        if key not in lookup:
            raise AssertionError(f"tree edge {key} is not a candidate")
        in_edge[v] = lookup[key]
    return emit(ptr, idx, f, in_edge), (f, t, w)


def spmm_update(row_ptr, col, val, x, branches, src, dst, parallel=False):
    """s_spmm_update_csr_int32 (cbm/cbm_extensions.cpp:351-444) / matmul_AX_ADX in fp32."""
    x = _c(x, np.float32)
    n = row_ptr.size - 1
    c = x.shape[1]
    y = np.empty((n, c), np.float32)
    rp, ci, va = _c(row_ptr, np.int32), _c(col, np.int32), _c(val, np.float32)
    br, s, d = _c(branches, np.int32), _c(src, np.int32), _c(dst, np.int32)
    fn = lib().oracle_spmm_update_omp if parallel else lib().oracle_spmm_update
    fn(n, c, rp.ctypes.data, ci.ctypes.data, va.ctypes.data, x.ctypes.data, max(br.size - 1, 0), br.ctypes.data,
       s.ctypes.data, d.ctypes.data, y.ctypes.data)
    return y


def spmm_update_add(row_ptr, col, val, x, eps, branches, src, dst):
    """s_spmm_update_add_csr_int32 (cbm/cbm_extensions.cpp:498-591) in fp32: A x + (1 + eps) x."""
    x = _c(x, np.float32)
    n = row_ptr.size - 1
    c = x.shape[1]
    y = np.empty((n, c), np.float32)
    rp, ci, va = _c(row_ptr, np.int32), _c(col, np.int32), _c(val, np.float32)
    br, s, d = _c(branches, np.int32), _c(src, np.int32), _c(dst, np.int32)
    L = lib()
    L.oracle_spmm_update_add.restype = None
    L.oracle_spmm_update_add.argtypes = [i64, i64, vp, vp, vp, vp, C.c_float, i64, vp, vp, vp, vp]
    L.oracle_spmm_update_add(n, c, rp.ctypes.data, ci.ctypes.data, va.ctypes.data, x.ctypes.data, float(eps),
                             max(br.size - 1, 0), br.ctypes.data, s.ctypes.data, d.ctypes.data, y.ctypes.data)
    return y


def spmm_fused_update(row_ptr, col, val, x, branches, src, dst, mult, gpu_order=True, parallel=False):
    """matmul_DAX_DADX (cbm/cbm.cu:210-268; gpu_order) or s_spmm_fused_update_csr_int32
    (cbm/cbm_extensions.cpp:593-698) in fp32."""
    x = _c(x, np.float32)
    n = row_ptr.size - 1
    c = x.shape[1]
    y = np.empty((n, c), np.float32)
    rp, ci, va = _c(row_ptr, np.int32), _c(col, np.int32), _c(val, np.float32)
    br, s, d, m = _c(branches, np.int32), _c(src, np.int32), _c(dst, np.int32), _c(mult, np.float32)
    if parallel:
        lib().oracle_spmm_fused_update_omp(n, c, rp.ctypes.data, ci.ctypes.data, va.ctypes.data, x.ctypes.data,
                                           max(br.size - 1, 0), br.ctypes.data, s.ctypes.data, d.ctypes.data,
                                           m.ctypes.data, y.ctypes.data)
    else:
        lib().oracle_spmm_fused_update(n, c, rp.ctypes.data, ci.ctypes.data, va.ctypes.data, x.ctypes.data,
                                       max(br.size - 1, 0), br.ctypes.data, s.ctypes.data, d.ctypes.data,
                                       m.ctypes.data, 0 if gpu_order else 1, y.ctypes.data)
    return y


def dense_f64(ptr, idx, n_cols, x, rs=None, cs=None, transpose=False):
    """FP64 y = rs o (A (cs o x)) (or A^T) over the binary pattern of A."""
    x = _c(x, np.float64)
    n_rows = ptr.size - 1
    c = x.shape[1]
    out_rows = n_cols if transpose else n_rows
    y = np.empty((out_rows, c), np.float64)
    ptr, idx = _c(ptr, np.int64), _c(idx, np.int32)
    rs_ = _c(rs, np.float64) if rs is not None else None
    cs_ = _c(cs, np.float64) if cs is not None else None
    lib().oracle_csr_spmm_f64(n_rows, n_cols, ptr.ctypes.data, idx.ctypes.data, c, x.ctypes.data,
                              rs_.ctypes.data if rs_ is not None else None,
                              cs_.ctypes.data if cs_ is not None else None, int(transpose), y.ctypes.data)
    return y


def degree_inv_sqrt(ptr):
    """D^-1/2 of the row degrees, fp32 then fp64 (as the classes compute it)."""
    d = np.diff(ptr).astype(np.float32)
    with np.errstate(divide="ignore"):
        return (1.0 / np.sqrt(d.astype(np.float64))).astype(np.float64)


def threads():
    return int(lib().oracle_threads())


# ---- the reference's cbm_mkl_cpp products (cbm/cbm_extensions.cpp:351-907) ------
# Same names, argument order and in-place ``dst`` as the reference's operators,
# on numpy arrays; each composes the C pieces as the reference composes MKL's
# SpMM, the branch-serial update and cblas_saxpy.

def _mkl_lib():
    L = lib()
    if not getattr(L, "_mkl_ready", False):
        L.oracle_spmm_be.restype = None
        L.oracle_spmm_be.argtypes = [i64, i64, vp, vp, vp, vp, vp, vp]
        L.oracle_spmm_t_be.restype = None
        L.oracle_spmm_t_be.argtypes = [i64, i64, i64, vp, vp, vp, vp, vp, vp]
        L.oracle_update_only.restype = None
        L.oracle_update_only.argtypes = [i64, i64, vp, vp, vp, vp, i32, vp]
        L.oracle_axpy.restype = None
        L.oracle_axpy.argtypes = [i64, C.c_float, vp, vp]
        L._mkl_ready = True
    return L


def _out(dst):
    if not (isinstance(dst, np.ndarray) and dst.dtype == np.float32 and dst.flags.c_contiguous and dst.ndim == 2):
        raise TypeError("dst must be a C-contiguous float32 numpy matrix")
    return dst


def _spmm_into(rp_b, rp_e, col, val, rhs, dst):
    rp_b, rp_e, col = _c(rp_b, np.int32), _c(rp_e, np.int32), _c(col, np.int32)
    val, rhs = _c(val, np.float32), _c(rhs, np.float32)
    _mkl_lib().oracle_spmm_be(dst.shape[0], dst.shape[1], rp_b.ctypes.data, rp_e.ctypes.data, col.ctypes.data,
                              val.ctypes.data, rhs.ctypes.data, dst.ctypes.data)
    return rhs


def _update_into(branches, src, dst_idx, mult, mode, dst):
    br, s, d = _c(branches, np.int32), _c(src, np.int32), _c(dst_idx, np.int32)
    m = _c(mult, np.float32) if mult is not None else None
    _mkl_lib().oracle_update_only(dst.shape[1], max(br.size - 1, 0), br.ctypes.data, s.ctypes.data, d.ctypes.data,
                                  m.ctypes.data if m is not None else None, mode, dst.ctypes.data)


def _axpy_into(a, rhs, dst):
    _mkl_lib().oracle_axpy(dst.size, float(a), rhs.ctypes.data, dst.ctypes.data)


def s_spmm_update_csr_int32(rp_b, rp_e, col, val, rhs, branches, src, dst_idx, dst):
    _spmm_into(rp_b, rp_e, col, val, rhs, _out(dst))
    _update_into(branches, src, dst_idx, None, 0, dst)


def s_spmm_fused_update_csr_int32(rp_b, rp_e, col, val, rhs, branches, src, dst_idx, multiplier, dst):
    _spmm_into(rp_b, rp_e, col, val, rhs, _out(dst))
    _update_into(branches, src, dst_idx, multiplier, 2, dst)


def s_spmm_add_csr_int32(rp_b, rp_e, col, val, rhs, eps, dst):
    x = _spmm_into(rp_b, rp_e, col, val, rhs, _out(dst))
    _axpy_into(np.float32(1.0) + np.float32(eps), x, dst)


def s_spmm_update_add_csr_int32(rp_b, rp_e, col, val, rhs, eps, branches, src, dst_idx, dst):
    x = _spmm_into(rp_b, rp_e, col, val, rhs, _out(dst))
    _update_into(branches, src, dst_idx, None, 0, dst)
    _axpy_into(np.float32(1.0) + np.float32(eps), x, dst)


def s_spmm_csr_int32(rp_b, rp_e, col, val, rhs, dst):
    _spmm_into(rp_b, rp_e, col, val, rhs, _out(dst))


def s_spmm_csr_t_int32(rp_b, rp_e, col, val, rhs, dst):
    rp_b, rp_e, col = _c(rp_b, np.int32), _c(rp_e, np.int32), _c(col, np.int32)
    val, rhs = _c(val, np.float32), _c(rhs, np.float32)
    _out(dst)
    _mkl_lib().oracle_spmm_t_be(rp_b.size, dst.shape[0], dst.shape[1], rp_b.ctypes.data, rp_e.ctypes.data,
                                col.ctypes.data, val.ctypes.data, rhs.ctypes.data, dst.ctypes.data)


def s_update_csr_int32(branches, src, dst_idx, dst):
    _update_into(branches, src, dst_idx, None, 0, _out(dst))


def s_fused_update_csr_int32(branches, src, dst_idx, multiplier, dst):
    _update_into(branches, src, dst_idx, multiplier, 2, _out(dst))
