"""Edge cases of the product path: the smallest graphs, zero columns, wide
operands split across column blocks, every row in one tree level or one
chain, the drop-in class with its reference-prepared values, and the
adjoint on the same shapes.  Each against the oracle (bit for bit where the
order of summation is the oracle's) or FP64."""
import numpy as np
import pytest
import torch

from conftest import chain_graph, near_dup_graph

pytestmark = pytest.mark.gpu


def _make(op, ei, alpha=0):
    from cbm import cbm4ad, cbm4dad, cbm4mm

    cls = {"ax": cbm4mm.cbm4mm, "adx": cbm4ad.cbm4ad, "dadx": cbm4dad.cbm4dad}[op]
    return cls(torch.from_numpy(np.ascontiguousarray(ei, dtype=np.int32)), torch.ones(ei.shape[1]), alpha=alpha)


def _oracle(op, a, x):
    from oracle import oracle

    args = (a.deltas.crow_indices().cpu().numpy(), a.deltas.col_indices().cpu().numpy(),
            a.deltas.values().cpu().numpy(), x.float().cpu().numpy(), a.mca_offset.cpu().numpy(),
            a.mca_src_idx.cpu().numpy(), a.mca_dst_idx.cpu().numpy())
    if op == "dadx":
        return oracle.spmm_fused_update(*args, a.D.cpu().numpy(), gpu_order=True)
    return oracle.spmm_update(*args)


@pytest.mark.parametrize("op", ["ax", "adx", "dadx"])
def test_two_node_graph(op):
    ei = np.array([[0, 1], [1, 0]])
    a = _make(op, ei)
    x = torch.tensor([[1.0, 2.0, 3.0, 4.0], [5.0, 6.0, 7.0, 8.0]], device="cuda")
    y = torch.empty_like(x)
    a.matmul(x, y)
    np.testing.assert_array_equal(y.cpu().numpy(), x.flip(0).cpu().numpy())  # D = 1: A x swaps the rows


def test_zero_columns_is_a_no_op():
    a = _make("ax", near_dup_graph(200, seed=3))
    x = torch.empty(200, 0, device="cuda")
    y = torch.empty(200, 0, device="cuda")
    a.matmul(x, y)
    a.plan.check_device()


@pytest.mark.parametrize("cols,dtype", [(2048, torch.float32), (2100, torch.float32), (4096, torch.bfloat16)])
def test_wide_operands_span_column_blocks(cols, dtype):
    a = _make("dadx", near_dup_graph(700, seed=7))
    x = torch.randn(700, cols, device="cuda").to(dtype)
    y = torch.empty(700, cols, device="cuda")
    a.matmul(x, y)
    np.testing.assert_array_equal(y.cpu().numpy(), _oracle("dadx", a, x))


def test_star_graph_one_hub_row_split_and_one_level():
    """One hub adjacent to every node: the hub's row is split in chunks, and
    the other rows are all equal (one entry each), so their delta rows are
    empty and their values come down the tree."""
    n = 5000
    leaves = np.arange(1, n)
    ei = np.concatenate([np.stack([np.zeros_like(leaves), leaves]), np.stack([leaves, np.zeros_like(leaves)])], 1)
    ei = ei[:, np.lexsort((ei[1], ei[0]))]
    a = _make("ax", ei)
    a.plan.tune(chunk_nnz=256)
    assert a.plan.stats["chunks"] > 0
    x = torch.randn(n, 64, device="cuda")
    y = torch.empty_like(x)
    a.matmul(x, y)
    ref = _oracle("ax", a, x)
    out = y.cpu().numpy()
    np.testing.assert_array_equal(out[1:], ref[1:])  # unsplit rows: the oracle's order
    np.testing.assert_allclose(out[0], x[1:].sum(0).cpu().numpy(), rtol=1e-4, atol=1e-3)


@pytest.mark.parametrize("variant", ["auto", "register", "tma"])
def test_deep_chain_adjoint_and_forward(variant):
    ei, n = chain_graph(700)
    a = _make("ax", ei)
    a.plan.tune(variant=variant)
    x = torch.randn(n, 64, device="cuda")
    y = torch.empty_like(x)
    a.matmul(x, y)
    np.testing.assert_array_equal(y.cpu().numpy(), _oracle("ax", a, x))
    g = torch.randn(n, 64, device="cuda")
    dx = torch.empty_like(g)
    a.adjoint(g, dx)
    a.plan.check_device()
    # A^T g for the chain: column n + j is held by rows j..n-1
    gg = g.double().cpu().numpy()
    ref = np.zeros((n, 64))
    ref[n // 2:] = np.cumsum(gg[: n // 2][::-1], axis=0)[::-1]
    assert np.abs(dx.double().cpu().numpy() - ref).max() <= 1e-4 * max(1.0, np.abs(ref).max())
