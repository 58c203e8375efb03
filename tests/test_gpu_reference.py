"""Parity with the reference's own GPU path (cbm/cbm.cu compiled from the
reference sources into oracle/_ref/ by oracle/build_ref.py) on the same
structure, and a pin of the oracle against it.

Tolerance rtol 1e-5, atol 1e-6: cuSPARSE's SpMM sums a row in an order of its
own choosing, so the reference and this library agree to rounding, not bit
for bit.

Harness note: the reference launches one block per entry of mca_branches,
i.e. B + 1 blocks for B branches (cbm/cbm.cu:136, :193), and the last block
reads mca_branches[B + 1], one element past the tensor.  The tensor handed to
it here is a view of a buffer with one more element equal to the edge count,
so that read finds an empty range.

Set CBM_REF_TIMING=1 to also time both paths on the 1M-node DAD workload
(CBM_REF_TIMING_OUT=path also writes the record there as JSON).
"""
import os
import time

import numpy as np
import pytest
import torch

from conftest import near_dup_graph, random_graph

pytestmark = pytest.mark.gpu
RTOL, ATOL = 1e-5, 1e-6


@pytest.fixture(scope="module")
def ref_mod():
    from oracle import build_ref

    mod = build_ref.load("cbm_cusparse_ref")
    if mod is None:
        pytest.skip("reference GPU module not built (oracle/_ref/cbm_cusparse_ref.so)")
    return mod


def _prepare(ei, alpha):
    """Structure prepared exactly as the reference classes do (cbm/cbm4mm.py:9-51,
    cbm/cbm4dad.py:7-51), plus this library's cbm4dad on the same graph."""
    from cbm.cbm4dad import cbm4dad

    dev = torch.device("cuda")
    ours = cbm4dad(torch.from_numpy(ei), torch.ones(ei.shape[1]), alpha=alpha)
    n = ours.num_nodes
    crow = ours.deltas.crow_indices()
    col = ours.deltas.col_indices()
    signs = torch.from_numpy(__import__("cbm.cbm_mkl_cpp", fromlist=["x"]).build(ei[0], ei[1], n, alpha).csr_val)
    signs = signs.to(dev)
    br = ours.mca_offset
    br_pad = torch.cat([br, br[-1:]])[: br.numel()]  # one readable sentinel past the end
    return ours, n, crow, col, signs, br_pad, dev


@pytest.mark.parametrize("graph", ["near_dup", "random", "community"])
def test_ax_and_dadx_match_reference(graph, ref_mod):
    if graph == "near_dup":
        ei = near_dup_graph(3000, seed=31, deg=14)
    elif graph == "random":
        ei = random_graph(2500, 10, seed=8)
    else:
        from cbm.synthetic import workload

        ei = workload("community-4096")[0]
    ours, n, crow, col, signs, br_pad, dev = _prepare(ei, 0)
    src, dst = ours.mca_src_idx, ours.mca_dst_idx
    plain = torch.sparse_csr_tensor(crow, col, signs, (n, n))
    empty = torch.empty(0, device=dev)
    ref_ax = ref_mod.cusparseCBM(plain, br_pad, src, dst, empty)
    x = torch.rand(n, 128, device=dev)
    y_ref = torch.empty_like(x)
    assert ref_ax.matmul_AX_ADX(x, y_ref) == 0
    y = torch.empty_like(x)
    ours.plan.matmul("ax", x, y)
    torch.cuda.synchronize()
    torch.testing.assert_close(y, y_ref, rtol=RTOL, atol=ATOL)

    # DAD: values and multipliers as cbm4dad prepares them
    dad = torch.sparse_csr_tensor(crow, col, ours.deltas.values(), (n, n))
    ref_dad = ref_mod.cusparseCBM(dad, br_pad, src, dst, ours.D)
    y_ref2 = torch.empty_like(x)
    assert ref_dad.matmul_DAX_DADX(x, y_ref2) == 0
    y2 = torch.empty_like(x)
    ours.matmul(x, y2)
    torch.cuda.synchronize()
    torch.testing.assert_close(y2, y_ref2, rtol=RTOL, atol=ATOL)

    # the oracle agrees with the reference too (pins the oracle's restatement)
    from oracle import oracle

    o = oracle.spmm_fused_update(crow.cpu().numpy(), col.cpu().numpy(), ours.deltas.values().cpu().numpy(),
                                 x.cpu().numpy(), ours.mca_offset.cpu().numpy(), src.cpu().numpy(),
                                 dst.cpu().numpy(), ours.D.cpu().numpy())
    torch.testing.assert_close(torch.from_numpy(o), y_ref2.cpu(), rtol=RTOL, atol=ATOL)


def test_degree_through_reference_product(ref_mod):
    """The reference computes d = A 1 with its own product (cbm/cbm4dad.py:11-16): same D."""
    ei = near_dup_graph(2000, seed=5)
    ours, n, crow, col, signs, br_pad, dev = _prepare(ei, 0)
    ref = ref_mod.cusparseCBM(torch.sparse_csr_tensor(crow, col, signs, (n, n)), br_pad, ours.mca_src_idx,
                              ours.mca_dst_idx, torch.empty(0, device=dev))
    d = torch.zeros(n, 1, device=dev)
    ref.matmul_AX_ADX(torch.ones(n, 1, device=dev), d)
    assert torch.equal((d ** (-1 / 2)).view(-1), ours.D)


@pytest.mark.skipif(os.environ.get("CBM_REF_TIMING") != "1", reason="timing run only on request")
def test_time_reference_vs_ours(ref_mod):
    import json

    from cbm import synthetic

    ei, n, spec = synthetic.workload("powerlaw-1m")
    ours, n, crow, col, signs, br_pad, dev = _prepare(ei, spec["alpha"])
    ref = ref_mod.cusparseCBM(torch.sparse_csr_tensor(crow, col, ours.deltas.values(), (n, n)), br_pad,
                              ours.mca_src_idx, ours.mca_dst_idx, ours.D)
    x = torch.randn(n, 256, device=dev)
    y1, y2 = torch.empty_like(x), torch.empty_like(x)

    def timeit(fn, k=20):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(k):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k

    t_ref = timeit(lambda: ref.matmul_DAX_DADX(x, y1))
    t_ours = timeit(lambda: ours.matmul(x, y2))
    torch.testing.assert_close(y2, y1, rtol=RTOL, atol=ATOL)
    # the reference's CSR baseline (cbm/csr.cu) on D^-1/2 A D^-1/2 itself
    from oracle import build_ref, oracle

    csr_mod = build_ref.load("csr_cusparse_ref")
    t_csr = None
    if csr_mod is not None:
        ptr, idx = oracle.csr_from_edges(ei, n)
        rows = torch.repeat_interleave(torch.arange(n, device=dev), torch.from_numpy(np.diff(ptr)).to(dev))
        colt = torch.from_numpy(idx).to(dev)
        vals = ours.D[rows] * ours.D[colt.long()]
        ahat = torch.sparse_csr_tensor(torch.from_numpy(ptr.astype(np.int32)).to(dev), colt, vals, (n, n))
        csr = csr_mod.cusparseCSR(ahat)
        y3 = torch.empty_like(x)
        t_csr = timeit(lambda: csr.matmul(x, y3))
        torch.testing.assert_close(y3, y1, rtol=1e-4, atol=1e-5)
    st = ours.plan.stats
    from bench import bytes_alg

    b = bytes_alg(n, st["nnz"], st["edges"], st["branches"], 256)
    rec = {"workload": "powerlaw-1m dadx C=256", "ref_ms": t_ref, "ours_ms": t_ours, "ref_gbs": b / t_ref / 1e6,
           "ours_gbs": b / t_ours / 1e6, "speedup": t_ref / t_ours, "ref_csr_ms": t_csr,
           "speedup_vs_csr": (t_csr / t_ours) if t_csr else None, "when": time.time()}
    print("REFTIMING", json.dumps(rec))
    out = os.environ.get("CBM_REF_TIMING_OUT")
    if out:
        with open(out, "w") as f:
            json.dump(rec, f)
