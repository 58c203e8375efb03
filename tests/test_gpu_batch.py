"""Batching form: a block-diagonal CBM of many graphs in one launch equals the
graphs' own products bit for bit; CUDA-graph replay and the autotuner; and the
512-graph workload (log-uniform 1,000..64,000 nodes, mean degree U[8, 40],
BF16 X with 64 columns, seed 4) replayed from a CUDA graph against the oracle
(each sampled graph's slice bit for bit) and against FP64 on sampled rows."""
import numpy as np
import pytest
import torch

from conftest import near_dup_graph

pytestmark = pytest.mark.gpu


def _graphs(count=12, seed=0):
    from cbm import synthetic

    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.integers(200, 3000))
        if i % 3 == 0:
            ei = near_dup_graph(n, seed=100 + i, deg=8)
        else:
            ei = synthetic.community_graph(n, 64, int(rng.integers(4, 12)), 2, seed=200 + i)
        out.append((ei, n))
    return out


@pytest.mark.parametrize("op,xdt", [("dadx", torch.bfloat16), ("ax", torch.float32), ("adx", torch.float32)])
def test_batch_matches_single_graphs(op, xdt):
    from cbm.batch import cbm_batch
    from cbm.cbm4ad import cbm4ad
    from cbm.cbm4dad import cbm4dad
    from cbm.cbm4mm import cbm4mm

    graphs = _graphs()
    b = cbm_batch(graphs, alpha=0, op=op)
    x = torch.randn(b.num_nodes, 64, device="cuda").to(xdt)
    y = torch.empty(b.num_nodes, 64, device="cuda")
    b.matmul(x, y)
    cls = {"ax": cbm4mm, "adx": cbm4ad, "dadx": cbm4dad}[op]
    for (ei, n), xs, ys in zip(graphs, b.split(x), b.split(y)):
        single = cls(torch.from_numpy(ei), torch.ones(ei.shape[1]), alpha=0)
        assert single.num_nodes == n
        yy = torch.empty(n, 64, device="cuda")
        single.matmul(xs.contiguous(), yy)
        assert torch.equal(ys, yy)
    b.plan.check_device()


def test_batch_graph_replay_and_autotune():
    from cbm.batch import cbm_batch
    from cbm.tune import autotune

    graphs = _graphs(20, seed=1)
    b = cbm_batch(graphs, alpha=0, op="dadx")
    x = torch.randn(b.num_nodes, 64, device="cuda").to(torch.bfloat16)
    y = torch.empty(b.num_nodes, 64, device="cuda")
    ref = torch.empty_like(y)
    b.matmul(x, ref)
    res = autotune(b.plan, "dadx", x, y, space={"chunk_nnz": [64, 256], "rows_per_claim": [1, 4],
                                                  "variant": ["auto", "register"]})
    assert len(res) == 8 and res[0][1] <= res[-1][1]
    g = b.capture(x, y)
    for seed in range(3):
        x.copy_(torch.randn(b.num_nodes, 64, device="cuda", generator=torch.Generator(device="cuda").manual_seed(seed)))
        g.replay()
        b.matmul(x, ref)
        torch.cuda.synchronize()
        # tuning may change how long rows are split: equal to rounding
        torch.testing.assert_close(y, ref, rtol=1e-5, atol=1e-6)
    b.plan.check_device()


@pytest.fixture(scope="module")
def batch512():
    from cbm import synthetic
    from cbm.batch import cbm_batch

    graphs = synthetic.batch_graphs(512, seed=4)
    return graphs, cbm_batch(graphs, alpha=0, op="dadx")


def test_batch512_vs_oracle(batch512):
    """One launch of D^-1/2 A D^-1/2 X over all 512 graphs, replayed from a CUDA
    graph; every sampled graph's rows equal the oracle's
    s_spmm_fused_update restatement with the reference GPU's propagation
    rounding (cbm/cbm.cu:59-91) on that graph's own structure."""
    import bench
    from oracle import oracle

    graphs, b = batch512
    n = b.num_nodes
    assert len(graphs) == 512 and n > 8_000_000
    g = torch.Generator(device="cuda").manual_seed(4)
    x = torch.randn(n, 64, device="cuda", generator=g).to(torch.bfloat16)
    y = torch.full((n, 64), float("nan"), device="cuda")
    replay = b.capture(x, y)
    y.fill_(float("nan"))
    replay.replay()
    torch.cuda.synchronize()
    b.plan.check_device()
    st = b.plan.stats
    # no row is long enough to be split, so every row sums in the oracle's order
    assert st["chunks"] == 0, st
    rng = np.random.default_rng(4)
    sizes = np.array(b.sizes)
    pick = set(rng.choice(len(graphs), 40, replace=False).tolist()) | {int(sizes.argmin()), int(sizes.argmax())}
    dd = b.D.cpu().numpy()
    for gi in sorted(pick):
        crow, col, val, br, src, dst = b.graph_structure(gi)
        off, end = int(b.offsets[gi]), int(b.offsets[gi + 1])
        d = dd[off:end]
        rows = np.repeat(np.arange(end - off), np.diff(crow))
        pval = (val * d[col]) * d[rows]  # the entry scale the kernel forms: (s D[col]) D[row]
        ref = oracle.spmm_fused_update(crow, col, pval, x[off:end].float().cpu().numpy(), br, src, dst, d,
                                       gpu_order=True)
        out = y[off:end].cpu().numpy()
        assert np.array_equal(out, ref), (gi, float(np.nanmax(np.abs(out - ref))))
    # the whole batch (every graph) against FP64 sums over the original edges
    packed = np.concatenate([np.asarray(ei, dtype=np.int64) + int(b.offsets[i]) for i, (ei, _) in enumerate(graphs)],
                            axis=1)
    dinv = bench.dinv_f64(packed, n)
    err = bench.fp64_sample_error(packed, n, x, y, rs=dinv, cs=dinv, rows=16384, seed=4)
    print("512-graph batch vs FP64:", err)
    assert err["max_rel"] <= 1e-5 and err["rel_fro"] <= 1e-6
    assert not torch.isnan(y).any()
