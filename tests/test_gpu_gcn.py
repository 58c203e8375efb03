"""The differentiation form: a 2-layer GCN through cbm4dad's autograd products.

* full 170,000-node workload: logits and weight gradients of the BF16 and FP32
  forms against an FP64 forward/backward built from the oracle's FP64 products
  (relative error = ||ours - ref|| / ||ref||, Frobenius; BF16 bar 1e-2);
* a 2,000-node induced subgraph: gradients against torch autograd over a dense
  FP64 adjacency, and a directional finite-difference check.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _ahat64(ptr, idx, dinv, m):
    from oracle import oracle

    return oracle.dense_f64(ptr, idx, ptr.size - 1, m, rs=dinv, cs=dinv)


def _reference(ei, n, x64, w1, w2, labels):
    """FP64 logits and weight gradients of mean cross-entropy."""
    from oracle import oracle

    ptr, idx = oracle.csr_from_edges(ei, n)
    deg = np.diff(ptr).astype(np.float64)
    with np.errstate(divide="ignore"):
        dinv = 1.0 / np.sqrt(deg)
    dinv[deg == 0] = 0.0
    ax = _ahat64(ptr, idx, dinv, x64)
    z1 = ax @ w1
    h = np.maximum(z1, 0.0)
    hw = h @ w2
    logits = _ahat64(ptr, idx, dinv, hw)
    p = np.exp(logits - logits.max(axis=1, keepdims=True))
    p /= p.sum(axis=1, keepdims=True)
    p[np.arange(n), labels] -= 1.0
    dl = p / n
    dhw = _ahat64(ptr, idx, dinv, dl)  # Ahat is symmetric
    dw2 = h.T @ dhw
    dz1 = (dhw @ w2.T) * (z1 > 0)
    dw1 = ax.T @ dz1
    return logits, dw1, dw2, dhw


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def gcn_graph():
    from cbm import synthetic
    from cbm.cbm4dad import cbm4dad

    ei, n, spec = synthetic.workload("powerlaw-170k")
    a = cbm4dad(torch.from_numpy(ei), torch.ones(ei.shape[1]), alpha=spec["alpha"])
    return ei, n, a


@pytest.mark.parametrize("dtype,bar", [(torch.bfloat16, 1e-2), (torch.float32, 1e-5)])
def test_gcn_against_fp64(gcn_graph, dtype, bar):
    from cbm.gcn import GCN

    ei, n, a = gcn_graph
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn(n, 128, device="cuda", generator=g).to(dtype)
    labels = torch.randint(0, 40, (n,), device="cuda", generator=g)
    model = GCN(a, 128, 256, 40, act_dtype=dtype)
    seen = {}
    logits = model(x)
    # the CBM adjoint's output: the gradient reaching H W2 through Ahat^T
    hw_node = logits.grad_fn
    hw_node.register_hook(lambda gin, gout: seen.__setitem__("dhw", gin[0]))
    loss = torch.nn.functional.cross_entropy(logits, labels)
    loss.backward()
    ref_logits, ref_dw1, ref_dw2, ref_dhw = _reference(
        ei, n, x.double().cpu().numpy(), model.w1.detach().double().cpu().numpy(),
        model.w2.detach().double().cpu().numpy(), labels.cpu().numpy())
    errs = {"logits (forward)": _rel(logits.detach().double().cpu().numpy(), ref_logits),
            "Ahat^T G (adjoint)": _rel(seen["dhw"].double().cpu().numpy(), ref_dhw),
            "dW1": _rel(model.w1.grad.double().cpu().numpy(), ref_dw1),
            "dW2": _rel(model.w2.grad.double().cpu().numpy(), ref_dw2)}
    print(f"GCN {dtype} relative error vs FP64:", errs)
    # the bar holds for the CBM layer's forward and adjoint products; the
    # weight gradients add BF16 storage of activations and gradients summed
    # over 170,000 rows with heavy cancellation, so they get a looser check
    assert errs["logits (forward)"] <= bar and errs["Ahat^T G (adjoint)"] <= bar, errs
    assert errs["dW1"] <= 5 * bar and errs["dW2"] <= 5 * bar, errs
    a.plan.check_device()


def _bfs_subgraph(ei, n, size, start):
    nbrs = [[] for _ in range(n)]
    for u, v in zip(ei[0].tolist(), ei[1].tolist()):
        nbrs[u].append(v)
    seen = {start: 0}
    order = [start]
    i = 0
    while i < len(order) and len(order) < size:
        for w in nbrs[order[i]]:
            if w not in seen and len(order) < size:
                seen[w] = len(order)
                order.append(w)
        i += 1
    keep = np.array([u in seen and v in seen for u, v in zip(ei[0], ei[1])])
    sub = np.stack([[seen[u] for u in ei[0][keep]], [seen[v] for v in ei[1][keep]]]).astype(np.int32)
    return sub, len(order)


def test_gcn_gradients_on_2000_node_subgraph(gcn_graph):
    from cbm.cbm4dad import cbm4dad
    from cbm.gcn import GCN

    ei, n, _ = gcn_graph
    deg = np.bincount(ei[0], minlength=n)
    sub, m = _bfs_subgraph(ei, n, 2000, int(np.argmax(deg == np.median(deg[deg > 0]))))
    assert m == 2000
    a = cbm4dad(torch.from_numpy(sub), torch.ones(sub.shape[1]), alpha=0)
    m = a.num_nodes
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.randn(m, 128, device="cuda", generator=g)
    labels = torch.randint(0, 40, (m,), device="cuda", generator=g)
    model = GCN(a, 128, 256, 40, act_dtype=torch.float32, seed=7)

    def loss_of(w1, w2):
        # the same network on a dense FP64 adjacency, for torch autograd
        A = torch.zeros(m, m, dtype=torch.float64, device="cuda")
        A[torch.from_numpy(sub[0]).long(), torch.from_numpy(sub[1]).long()] = 1.0
        dinv = A.sum(1).pow(-0.5)
        dinv[torch.isinf(dinv)] = 0
        ah = dinv[:, None] * A * dinv[None, :]
        h = torch.relu(ah @ x.double() @ w1)
        return torch.nn.functional.cross_entropy(ah @ (h @ w2), labels)

    loss = torch.nn.functional.cross_entropy(model(x), labels)
    loss.backward()
    w1 = model.w1.detach().double().clone().requires_grad_(True)
    w2 = model.w2.detach().double().clone().requires_grad_(True)
    ref = loss_of(w1, w2)
    ref.backward()
    assert abs(loss.item() - ref.item()) <= 1e-5 * abs(ref.item())
    assert _rel(model.w1.grad.double().cpu().numpy(), w1.grad.cpu().numpy()) <= 1e-4
    assert _rel(model.w2.grad.double().cpu().numpy(), w2.grad.cpu().numpy()) <= 1e-4
    # directional finite differences of the CBM model's loss (the loss reduced
    # in FP64 from the model's fp32 logits), along the gradient and along a
    # random direction mixed with it
    g1, g2 = model.w1.grad.detach().clone(), model.w2.grad.detach().clone()
    scale = 1.0 / float(torch.sqrt((g1 * g1).sum() + (g2 * g2).sum()))
    for seed in range(2):
        gd = torch.Generator(device="cuda").manual_seed(100 + seed)
        d1 = g1 * scale + (0.5 * seed) * torch.randn(g1.shape, device="cuda", generator=gd) / g1.numel() ** 0.5
        d2 = g2 * scale + (0.5 * seed) * torch.randn(g2.shape, device="cuda", generator=gd) / g2.numel() ** 0.5
        h = 1e-2
        with torch.no_grad():
            w1c, w2c = model.w1.detach().clone(), model.w2.detach().clone()
            model.w1.copy_(w1c + h * d1)
            model.w2.copy_(w2c + h * d2)
            lp = torch.nn.functional.cross_entropy(model(x).double(), labels)
            model.w1.copy_(w1c - h * d1)
            model.w2.copy_(w2c - h * d2)
            lm = torch.nn.functional.cross_entropy(model(x).double(), labels)
            model.w1.copy_(w1c)
            model.w2.copy_(w2c)
        fd = (lp - lm) / (2 * h)
        an = (g1.double() * d1.double()).sum() + (g2.double() * d2.double()).sum()
        assert abs(fd - an) <= 1e-2 * abs(an), (fd.item(), an.item())
