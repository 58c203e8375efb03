"""GIN form Y = A X + (1 + eps) X (the reference's CPU-only
s_spmm_update_add_csr_int32, cbm/cbm_extensions.cpp:498-591).

CPU: the oracle's restatement against an FP64 product of the original A.
GPU: cbm4mm.matmul_add against the oracle, bit for bit (the self term is
fused into the final store as one fma per element; the rows propagated down
the tree are the A X rows)."""
import numpy as np
import pytest
import torch

from conftest import chain_graph, near_dup_graph, random_graph


def _structure(ei, n):
    from cbm import cbm_mkl_cpp

    return cbm_mkl_cpp.build(ei[0], ei[1], n, 0)


@pytest.mark.parametrize("eps", [0.0, 0.25, -1.5])
def test_oracle_gin_against_fp64(eps, oracle_mod):
    ei = near_dup_graph(800, seed=21)
    n = 800
    s = _structure(ei, n)
    x = np.random.default_rng(2).standard_normal((n, 24)).astype(np.float32)
    y = oracle_mod.spmm_update_add(s.csr_ptr, s.csr_col, s.csr_val, x, eps, s.branches, s.src, s.dst)
    ptr, idx = oracle_mod.csr_from_edges(ei, n)
    ref = oracle_mod.dense_f64(ptr, idx, n, x.astype(np.float64)) + (1.0 + eps) * x.astype(np.float64)
    assert np.abs(y - ref).max() <= 1e-5 * max(1.0, np.abs(ref).max())


def _gpu_case(ei, n, cols, dtype, eps, variant, ydt=torch.float32):
    from cbm.cbm4mm import cbm4mm
    from oracle import oracle

    a = cbm4mm(torch.from_numpy(ei), torch.ones(ei.shape[1]), alpha=0)
    a.plan.tune(variant=variant)
    x = torch.randn(a.num_nodes, cols, device="cuda").to(dtype)
    y = torch.empty(a.num_nodes, cols, device="cuda", dtype=ydt)
    a.matmul_add(x, y, eps)
    a.plan.check_device()
    ref = oracle.spmm_update_add(a.deltas.crow_indices().cpu().numpy(), a.deltas.col_indices().cpu().numpy(),
                                 a.deltas.values().cpu().numpy(), x.float().cpu().numpy(), eps,
                                 a.mca_offset.cpu().numpy(), a.mca_src_idx.cpu().numpy(),
                                 a.mca_dst_idx.cpu().numpy())
    return y, ref


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["register", "staged"])
@pytest.mark.parametrize("cols,dtype", [(64, torch.float32), (256, torch.float32), (128, torch.bfloat16),
                                        (40, torch.float32)])
def test_gin_matches_oracle(variant, cols, dtype):
    y, ref = _gpu_case(near_dup_graph(3000, seed=5, deg=14), 3000, cols, dtype, 0.3, variant)
    np.testing.assert_array_equal(y.cpu().numpy(), ref)


@pytest.mark.gpu
def test_gin_on_a_chain_and_random_graph():
    ei, n = chain_graph(300)
    # chain_graph is not square in its columns' use; matmul_add needs A square, which it is (2n x 2n)
    y, ref = _gpu_case(ei, n, 32, torch.float32, -0.5, "auto")
    np.testing.assert_array_equal(y.cpu().numpy(), ref)
    y, ref = _gpu_case(random_graph(2000, 9, seed=4), 2000, 64, torch.float32, 1.0, "auto")
    np.testing.assert_array_equal(y.cpu().numpy(), ref)


@pytest.mark.gpu
def test_gin_bf16_output_and_plain_product_unchanged():
    from cbm.cbm4mm import cbm4mm

    ei = near_dup_graph(2000, seed=8)
    y, ref = _gpu_case(ei, 2000, 128, torch.bfloat16, 0.1, "auto", ydt=torch.bfloat16)
    assert torch.equal(y.cpu(), torch.from_numpy(ref).to(torch.bfloat16))
    # the plain product on the same plan afterwards is untouched by the GIN call
    a = cbm4mm(torch.from_numpy(ei), torch.ones(ei.shape[1]), alpha=0)
    x = torch.randn(2000, 64, device="cuda")
    y1 = torch.empty_like(x)
    y2 = torch.empty_like(x)
    a.matmul(x, y1)
    a.matmul_add(x, y2, 0.0)
    a.matmul(x, y2)
    assert torch.equal(y1, y2)
