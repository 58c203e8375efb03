"""Batching form: a block-diagonal CBM of many graphs in one launch equals the
graphs' own products bit for bit; CUDA-graph replay and the autotuner."""
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
