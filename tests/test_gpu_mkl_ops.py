"""The reference's eight cbm_mkl_cpp products (cbm/cbm_extensions.cpp:351-907),
called with the reference's argument lists, against the oracle's restatement
of the same operators.

Rows sum their entries in order with one FMA each, the update and the GIN
term use the reference CPU path's arithmetic, so every operator but the
transposed product must equal the oracle bit for bit; the transposed product
adds with atomics (any order), so it is bounded by the magnitude of what was
summed.  Each operator runs on CUDA tensors (queued, errors read with
check_device) and on CPU tensors (the reference's own convention: copied to
the GPU and back, errors raised at once).
"""
import numpy as np
import pytest
import torch

from conftest import near_dup_graph

pytestmark = pytest.mark.gpu


def _structure(n=1500, seed=3):
    from cbm import cbm_mkl_cpp

    ei = near_dup_graph(n, seed=seed, deg=12)
    s = cbm_mkl_cpp.build(ei[0], ei[1], n, 0)
    assert s.src.size > 0 and s.branches.size > 1
    return s


def _values(s, kind, rng):
    """Entry values: the +-1 signs, or signs times positive weights (the values
    cbm4ad prepares are of this form)."""
    if kind == "signs":
        return s.csr_val.copy()
    return (s.csr_val * rng.uniform(0.1, 2.0, s.csr_val.size)).astype(np.float32)


OPS = ["s_spmm_update_csr_int32", "s_spmm_fused_update_csr_int32", "s_spmm_add_csr_int32",
       "s_spmm_update_add_csr_int32", "s_spmm_csr_int32", "s_spmm_csr_t_int32", "s_update_csr_int32",
       "s_fused_update_csr_int32"]


def _args(op, s, val, x, mult, eps, out):
    """The reference's argument list of ``op`` (cbm/cbm_extensions.cpp:911-918)."""
    rp_b, rp_e = s.csr_ptr[:-1], s.csr_ptr[1:]
    csr = [rp_b, rp_e, s.csr_col, val]
    tree = [s.branches, s.src, s.dst]
    return {
        "s_spmm_update_csr_int32": csr + [x] + tree + [out],
        "s_spmm_fused_update_csr_int32": csr + [x] + tree + [mult, out],
        "s_spmm_add_csr_int32": csr + [x, eps, out],
        "s_spmm_update_add_csr_int32": csr + [x, eps] + tree + [out],
        "s_spmm_csr_int32": csr + [x, out],
        "s_spmm_csr_t_int32": csr + [x, out],
        "s_update_csr_int32": tree + [out],
        "s_fused_update_csr_int32": tree + [mult, out],
    }[op]


def _torch(a, device):
    if isinstance(a, np.ndarray):
        return torch.from_numpy(np.ascontiguousarray(a)).to(device)
    return a


@pytest.mark.parametrize("op", OPS)
@pytest.mark.parametrize("where", ["cuda", "cpu"])
@pytest.mark.parametrize("cols", [64, 37])
def test_operator_matches_oracle(op, where, cols):
    from cbm import cbm_mkl_cpp
    from oracle import oracle

    rng = np.random.default_rng(cols)
    s = _structure()
    n = s.csr_ptr.size - 1
    val = _values(s, "weights", rng)
    x = rng.standard_normal((n, cols)).astype(np.float32)
    mult = rng.uniform(0.05, 1.0, n).astype(np.float32)
    eps = 0.25
    # the update-only operators start from a given dst
    start = rng.standard_normal((n, cols)).astype(np.float32)
    ref = start.copy()
    getattr(oracle, op)(*_args(op, s, val, x, mult, eps, ref))
    dev = torch.device(where)
    out = _torch(start.copy(), dev)
    targs = [_torch(a, dev) if isinstance(a, np.ndarray) else a for a in _args(op, s, val, x, mult, eps, out)]
    getattr(cbm_mkl_cpp, op)(*targs)
    if where == "cuda":
        cbm_mkl_cpp.check_device()
    got = out.cpu().numpy()
    if op == "s_spmm_csr_t_int32":
        # |A|^T |x| bounds the rounding of any summation order
        mag = np.empty_like(ref)
        oracle.s_spmm_csr_t_int32(s.csr_ptr[:-1], s.csr_ptr[1:], s.csr_col, np.abs(val), np.abs(x), mag)
        assert np.all(np.abs(got - ref) <= 1e-5 * mag + 1e-6)
    else:
        assert np.array_equal(got, ref), float(np.abs(got - ref).max())


def test_operators_close_to_fp64():
    """The CBM operators give A x (and the ratio form D^-1/2 A D^-1/2 x) of the
    original binary A to within FP32 rounding."""
    from cbm import cbm_mkl_cpp
    from oracle import oracle

    n = 1500
    ei = near_dup_graph(n, seed=3, deg=12)
    s = cbm_mkl_cpp.build(ei[0], ei[1], n, 0)
    rng = np.random.default_rng(0)
    x = rng.standard_normal((n, 64)).astype(np.float32)
    ptr, idx = oracle.csr_from_edges(ei, n)
    y64 = oracle.dense_f64(ptr, idx, n, x.astype(np.float64))
    out = torch.empty(n, 64, device="cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    cbm_mkl_cpp.s_spmm_update_csr_int32(t(s.csr_ptr[:-1]), t(s.csr_ptr[1:]), t(s.csr_col), t(s.csr_val), t(x),
                                        t(s.branches), t(s.src), t(s.dst), out)
    cbm_mkl_cpp.check_device()
    assert np.abs(out.cpu().numpy() - y64).max() <= 1e-5 * max(1.0, np.abs(y64).max())
    # D^-1/2 A D^-1/2 x: values s D[col] D[row], fused update with D
    d = np.diff(ptr).astype(np.float64)
    dinv = np.where(d > 0, 1.0 / np.sqrt(np.maximum(d, 1)), 0.0)
    d32 = dinv.astype(np.float32)
    rows = np.repeat(np.arange(n), np.diff(s.csr_ptr))
    val = (s.csr_val * d32[s.csr_col]) * d32[rows]
    cbm_mkl_cpp.s_spmm_fused_update_csr_int32(t(s.csr_ptr[:-1]), t(s.csr_ptr[1:]), t(s.csr_col), t(val), t(x),
                                              t(s.branches), t(s.src), t(s.dst), t(d32), out)
    cbm_mkl_cpp.check_device()
    y64 = oracle.dense_f64(ptr, idx, n, x.astype(np.float64), rs=dinv, cs=dinv)
    assert np.abs(out.cpu().numpy() - y64).max() <= 1e-5 * max(1.0, np.abs(y64).max())


def test_four_array_csr_with_gaps():
    """MKL's four-array CSR lets rows' entry ranges leave gaps: only
    [rp_b[i], rp_e[i]) belongs to row i."""
    from cbm import cbm_mkl_cpp
    from oracle import oracle

    rng = np.random.default_rng(7)
    n, cols = 300, 48
    lens = rng.integers(0, 9, n)
    gaps = rng.integers(0, 4, n)
    rp_b = np.zeros(n, np.int32)
    pos = 0
    for i in range(n):
        pos += int(gaps[i])
        rp_b[i] = pos
        pos += int(lens[i])
    rp_e = (rp_b + lens).astype(np.int32)
    col = rng.integers(0, n, pos).astype(np.int32)
    val = rng.standard_normal(pos).astype(np.float32)
    x = rng.standard_normal((n, cols)).astype(np.float32)
    ref = np.empty((n, cols), np.float32)
    oracle.s_spmm_csr_int32(rp_b, rp_e, col, val, x, ref)
    out = torch.empty(n, cols)
    cbm_mkl_cpp.s_spmm_csr_int32(*(torch.from_numpy(a) for a in (rp_b, rp_e, col, val, x)), out)
    assert np.array_equal(out.numpy(), ref)


def test_empty_tree_zero_columns_and_one_column():
    from cbm import cbm_mkl_cpp
    from oracle import oracle

    s = _structure(400, seed=5)
    n = s.csr_ptr.size - 1
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    no_branch = t(np.zeros(1, np.int32))
    none = t(np.zeros(0, np.int32))
    for cols in (0, 1):
        x = np.random.default_rng(cols).standard_normal((n, cols)).astype(np.float32)
        out = torch.full((n, cols), 7.0, device="cuda")
        cbm_mkl_cpp.s_spmm_update_csr_int32(t(s.csr_ptr[:-1]), t(s.csr_ptr[1:]), t(s.csr_col), t(s.csr_val), t(x),
                                            no_branch, none, none, out)
        cbm_mkl_cpp.check_device()
        ref = np.empty((n, cols), np.float32)
        oracle.s_spmm_csr_int32(s.csr_ptr[:-1], s.csr_ptr[1:], s.csr_col, s.csr_val, x, ref)
        assert np.array_equal(out.cpu().numpy(), ref)


def test_reference_dtype_errors():
    """Dtype checks raise RuntimeError with the reference's CHECK_DTYPE text, in
    its order (rhs first)."""
    from cbm import cbm_mkl_cpp

    s = _structure(200, seed=1)
    n = s.csr_ptr.size - 1
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    x = torch.randn(n, 8, device="cuda")
    out = torch.empty(n, 8, device="cuda")
    with pytest.raises(RuntimeError, match='"rhs" is not a tensor of type "torch::kFloat32"'):
        cbm_mkl_cpp.s_spmm_update_csr_int32(t(s.csr_ptr[:-1]), t(s.csr_ptr[1:]), t(s.csr_col), t(s.csr_val),
                                            x.double(), t(s.branches), t(s.src), t(s.dst), out)
    with pytest.raises(RuntimeError, match='"lhs_col_idx" is not a tensor of type "torch::kInt32"'):
        cbm_mkl_cpp.s_spmm_csr_int32(t(s.csr_ptr[:-1]), t(s.csr_ptr[1:]), t(s.csr_col).long(), t(s.csr_val), x, out)
    with pytest.raises(RuntimeError, match="same device"):
        cbm_mkl_cpp.s_spmm_csr_int32(t(s.csr_ptr[:-1]), t(s.csr_ptr[1:]), t(s.csr_col), t(s.csr_val), x.cpu(), out)


def test_device_errors_are_reported_and_cleared():
    """A column index out of range and a node with two parents are recorded on
    the device (the bad entry skipped), raised by check_device, and cleared:
    the next call is exact."""
    from cbm import _lib, cbm_mkl_cpp
    from oracle import oracle

    s = _structure(300, seed=2)
    n = s.csr_ptr.size - 1
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    x = np.random.default_rng(0).standard_normal((n, 16)).astype(np.float32)
    out = torch.empty(n, 16, device="cuda")
    bad_col = s.csr_col.copy()
    bad_col[5] = n + 10
    cbm_mkl_cpp.s_spmm_csr_int32(t(s.csr_ptr[:-1]), t(s.csr_ptr[1:]), t(bad_col), t(s.csr_val), t(x), out)
    with pytest.raises(_lib.CbmError) as e:
        cbm_mkl_cpp.check_device()
    assert e.value.code == _lib.ERR_INDEX
    # a second parent for some child
    src, dst = s.src.copy(), s.dst.copy()
    src = np.concatenate([src, src[:1]])
    dst = np.concatenate([dst, dst[-1:]]).astype(np.int32)
    br = s.branches.copy()
    br[-1] += 1
    cbm_mkl_cpp.s_spmm_update_csr_int32(t(s.csr_ptr[:-1]), t(s.csr_ptr[1:]), t(s.csr_col), t(s.csr_val), t(x),
                                        t(br), t(src), t(dst), out)
    with pytest.raises(_lib.CbmError) as e:
        cbm_mkl_cpp.check_device()
    assert e.value.code == _lib.ERR_STRUCTURE
    # CPU tensors: the error raises at once
    with pytest.raises(_lib.CbmError):
        cbm_mkl_cpp.s_spmm_csr_int32(*(torch.from_numpy(a) for a in (s.csr_ptr[:-1].copy(), s.csr_ptr[1:].copy(),
                                                                     bad_col, s.csr_val, x)), torch.empty(n, 16))
    # the status was cleared: a correct call passes and is exact
    cbm_mkl_cpp.s_spmm_update_csr_int32(t(s.csr_ptr[:-1]), t(s.csr_ptr[1:]), t(s.csr_col), t(s.csr_val), t(x),
                                        t(s.branches), t(s.src), t(s.dst), out)
    cbm_mkl_cpp.check_device()
    ref = np.empty((n, 16), np.float32)
    oracle.s_spmm_update_csr_int32(s.csr_ptr[:-1], s.csr_ptr[1:], s.csr_col, s.csr_val, x, s.branches, s.src, s.dst,
                                   ref)
    assert np.array_equal(out.cpu().numpy(), ref)


@pytest.mark.parametrize("op", OPS)
def test_operator_matches_reference_cpu_module(op):
    """Against the reference's own MKL operators, compiled from its source
    (oracle/build_ref.py): rtol 1e-5, atol 1e-6 (the transposed product:
    bounded by the magnitude of what was summed)."""
    from cbm import cbm_mkl_cpp
    from oracle import build_ref, oracle

    ref_mod = build_ref.load(build_ref.CPU_MODULE)
    if ref_mod is None:
        pytest.skip("the reference's CPU module is not built")
    rng = np.random.default_rng(11)
    s = _structure(2000, seed=8)
    n = s.csr_ptr.size - 1
    val = _values(s, "weights", rng)
    x = rng.standard_normal((n, 96)).astype(np.float32)
    mult = rng.uniform(0.05, 1.0, n).astype(np.float32)
    start = rng.standard_normal((n, 96)).astype(np.float32)
    want = torch.from_numpy(start.copy())
    getattr(ref_mod, op)(*[torch.from_numpy(np.ascontiguousarray(a)) if isinstance(a, np.ndarray) else a
                           for a in _args(op, s, val, x, mult, 0.125, want)])
    out = torch.from_numpy(start.copy()).cuda()
    getattr(cbm_mkl_cpp, op)(*[_torch(a, "cuda") if isinstance(a, np.ndarray) else a
                               for a in _args(op, s, val, x, mult, 0.125, out)])
    cbm_mkl_cpp.check_device()
    got = out.cpu().numpy()
    if op == "s_spmm_csr_t_int32":
        mag = np.empty_like(start)
        oracle.s_spmm_csr_t_int32(s.csr_ptr[:-1], s.csr_ptr[1:], s.csr_col, np.abs(val), np.abs(x), mag)
        assert np.all(np.abs(got - want.numpy()) <= 2e-5 * mag + 1e-6)
    else:
        np.testing.assert_allclose(got, want.numpy(), rtol=1e-5, atol=1e-6)
