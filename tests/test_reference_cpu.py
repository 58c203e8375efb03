"""The reference's own CPU product operators (cbm/cbm_extensions.cpp:351-907,
compiled from the reference source by oracle/build_ref.py against the MKL
entry points libtorch_cpu exports) pin the oracle's restatement of them: on
the same inputs both give the same FP32 results.  CPU only; skipped where the
reference module was not built (no reference tree at build time).
"""
import zlib

import numpy as np
import pytest
import torch

from conftest import chain_graph, near_dup_graph


@pytest.fixture(scope="module")
def ref():
    from oracle import build_ref

    m = build_ref.load(build_ref.CPU_MODULE)
    if m is None:
        pytest.skip("the reference's CPU module is not built (oracle/build_ref.py)")
    return m


def test_mkl_known_answer():
    """MKL's sparse entry points answer a 3x3 SpMM, its transpose and a saxpy
    exactly through the project's declarations (LP64, enum values)."""
    from oracle import build_ref

    if build_ref.load(build_ref.CPU_MODULE) is None:
        pytest.skip("the reference's CPU module is not built")
    assert build_ref.mkl_kat()


def _case(name):
    from cbm import cbm_mkl_cpp, synthetic

    if name == "near_dup":
        n = 2500
        ei = near_dup_graph(n, seed=21, deg=12)
    elif name == "powerlaw":
        n = 6000
        ei = synthetic._w_powerlaw(n, 2.1, 14.0, 0.3, 0.1, 22)
    else:
        ei, n = chain_graph(300)
    s = cbm_mkl_cpp.build(ei[0], ei[1], n, 0)
    return s, n


OPS = ["s_spmm_update_csr_int32", "s_spmm_fused_update_csr_int32", "s_spmm_add_csr_int32",
       "s_spmm_update_add_csr_int32", "s_spmm_csr_int32", "s_spmm_csr_t_int32", "s_update_csr_int32",
       "s_fused_update_csr_int32"]


def _args(op, s, val, x, mult, eps, out):
    csr = [s.csr_ptr[:-1].copy(), s.csr_ptr[1:].copy(), s.csr_col, val]
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


@pytest.mark.parametrize("graph", ["near_dup", "powerlaw", "chain"])
@pytest.mark.parametrize("op", OPS)
def test_oracle_equals_reference_cpu_operator(ref, graph, op):
    from oracle import oracle

    s, n = _case(graph)
    rng = np.random.default_rng(zlib.crc32(f"{graph}/{op}".encode()))
    cols = 40
    val = (s.csr_val * rng.uniform(0.1, 2.0, s.csr_val.size)).astype(np.float32)
    x = rng.standard_normal((n, cols)).astype(np.float32)
    mult = rng.uniform(0.05, 1.0, n).astype(np.float32)
    start = rng.standard_normal((n, cols)).astype(np.float32)
    want = start.copy()
    getattr(oracle, op)(*_args(op, s, val, x, mult, 0.5, want))
    got = torch.from_numpy(start.copy())
    getattr(ref, op)(*[torch.from_numpy(a) if isinstance(a, np.ndarray) else a
                       for a in _args(op, s, val, x, mult, 0.5, got)])
    if op == "s_spmm_csr_t_int32":
        mag = np.empty_like(want)
        oracle.s_spmm_csr_t_int32(s.csr_ptr[:-1], s.csr_ptr[1:], s.csr_col, np.abs(val), np.abs(x), mag)
        assert np.all(np.abs(got.numpy() - want) <= 1e-5 * mag + 1e-6)
    else:
        # rtol 1e-5 / atol 1e-6, the bar the products are held to; on the
        # machines measured so far MKL's row sums equal the oracle's in-order
        # FMAs bit for bit
        np.testing.assert_allclose(got.numpy(), want, rtol=1e-5, atol=1e-6)
