"""GPU parity of the adjoint dX = A_op^T G (reverse propagation + transposed
delta gather) against an FP64 oracle, finite differences and torch.sparse.
The reference has no backward; A_op^T of each form is:
    ax:   A^T G            adx:  D A^T G           dadx: D A^T D G
"""
import numpy as np
import pytest
import torch

from conftest import chain_graph, near_dup_graph, random_graph

pytestmark = pytest.mark.gpu


def _make(op, ei, alpha=0):
    from cbm import cbm4ad, cbm4dad, cbm4mm

    cls = {"ax": cbm4mm.cbm4mm, "adx": cbm4ad.cbm4ad, "dadx": cbm4dad.cbm4dad}[op]
    return cls(torch.from_numpy(ei), torch.ones(ei.shape[1]), alpha=alpha)


def _adj_f64(op, ei, n, g):
    from oracle import oracle

    ptr, idx = oracle.csr_from_edges(ei, n)
    d = np.diff(ptr).astype(np.float64)
    with np.errstate(divide="ignore"):
        dinv = 1.0 / np.sqrt(d)
    dinv[d == 0] = 0.0  # an empty row's product is 0 (inf * 0 in exact form)
    # (rs A cs)^T g = cs A^T (rs g)
    rs = dinv if op == "dadx" else None
    cs = dinv if op in ("adx", "dadx") else None
    gg = g.double().cpu().numpy()
    if rs is not None:
        gg = gg * rs[:, None]
    return oracle.dense_f64(ptr, idx, n, gg, rs=cs, transpose=True)


@pytest.mark.parametrize("op", ["ax", "adx", "dadx"])
@pytest.mark.parametrize("directed", [False, True])
def test_adjoint_vs_fp64(op, directed):
    dev = torch.device("cuda")
    n = 2500
    if directed:
        ei = random_graph(n, 8, seed=5, symmetric=False)
        # near-duplicate rows on top so that the tree is not trivial
        from cbm.synthetic import near_duplicates

        ei = near_duplicates(ei, n, 0.3, 0.1, seed=1)
        # keep it directed: near_duplicates symmetrises, so drop a random half of (i, j), i > j
        keep = (ei[0] < ei[1]) | (np.arange(ei.shape[1]) % 2 == 0)
        ei = np.ascontiguousarray(ei[:, keep])
        if op != "ax":
            pytest.skip("D^-1/2 of a directed graph with empty rows is infinite")
    else:
        ei = near_dup_graph(n, seed=7)
    a = _make(op, ei)
    g = torch.randn(n, 96, device=dev)
    dx = torch.empty(n, 96, device=dev)
    a.adjoint(g, dx)
    ref = _adj_f64(op, ei, n, g)
    out = dx.cpu().numpy()
    err = np.abs(out - ref).max()
    assert err <= 1e-4 * max(1.0, np.abs(ref).max()), err
    a.plan.check_device()


def test_symmetric_adjoint_equals_forward():
    dev = torch.device("cuda")
    ei = near_dup_graph(3000, seed=2)
    a = _make("dadx", ei)
    g = torch.randn(3000, 64, device=dev)
    fwd = torch.empty_like(g)
    adj = torch.empty_like(g)
    a.matmul(g, fwd)
    a.adjoint(g, adj)
    torch.testing.assert_close(adj, fwd, rtol=1e-5, atol=1e-5)


def test_adjoint_split_rows_and_chain():
    dev = torch.device("cuda")
    ei, n = chain_graph(300)
    a = _make("ax", ei)
    a.plan.tune(chunk_nnz=32, rows_per_claim=1)
    g = torch.randn(n, 48, device=dev)
    dx = torch.empty_like(g)
    a.adjoint(g, dx)
    ref = _adj_f64("ax", ei, n, g)
    assert np.abs(dx.cpu().numpy() - ref).max() <= 1e-4 * np.abs(ref).max()
    a.plan.check_device()


def test_autograd_directional_finite_difference():
    """f(x) = <w, A x> is linear: (f(x + h d) - f(x - h d)) / 2h = <A^T w, d> exactly in
    real arithmetic; checked in fp32 on a 2,000-node graph."""
    dev = torch.device("cuda")
    ei = near_dup_graph(2000, seed=13)
    a = _make("dadx", ei)
    x = torch.randn(2000, 32, device=dev, requires_grad=True)
    w = torch.randn(2000, 32, device=dev)
    y = a.forward(x)
    (y * w).sum().backward()
    grad = x.grad.detach()
    for seed in range(3):
        d = torch.randn(2000, 32, device=dev, generator=torch.Generator(device=dev).manual_seed(seed))
        with torch.no_grad():
            fp = (a.forward(x + d) * w).double().sum()
            fm = (a.forward(x - d) * w).double().sum()
        fd = (fp - fm) / 2
        an = (grad.double() * d.double()).sum()
        assert abs(fd - an) <= 1e-4 * max(1.0, abs(an)), (fd, an)


def test_autograd_vs_torch_sparse():
    dev = torch.device("cuda")
    n = 1800
    ei = near_dup_graph(n, seed=21)
    a = _make("adx", ei)
    x = torch.randn(n, 40, device=dev, requires_grad=True)
    y = a.forward(x)
    w = torch.randn_like(y)
    (y * w).sum().backward()
    # torch.sparse reference of A D^-1/2 in fp64
    idx = torch.from_numpy(ei).long()
    A = torch.sparse_coo_tensor(idx, torch.ones(idx.shape[1], dtype=torch.float64), (n, n)).coalesce().to(dev)
    D = a.D.double()
    x64 = x.detach().double().requires_grad_(True)
    y64 = torch.sparse.mm(A, x64 * D[:, None])
    (y64 * w.double()).sum().backward()
    torch.testing.assert_close(y.double(), y64, rtol=1e-5, atol=1e-5)
    torch.testing.assert_close(x.grad.double(), x64.grad, rtol=1e-5, atol=1e-5)


def test_bf16_gradients():
    dev = torch.device("cuda")
    n = 2000
    ei = near_dup_graph(n, seed=4)
    a = _make("dadx", ei)
    x = torch.randn(n, 64, device=dev).to(torch.bfloat16).requires_grad_(True)
    y = a.forward(x)
    assert y.dtype == torch.bfloat16
    g = torch.randn(n, 64, device=dev).to(torch.bfloat16)
    y.backward(g)
    ref = _adj_f64("dadx", ei, n, g.float())
    rel = np.abs(x.grad.float().cpu().numpy() - ref).max() / np.abs(ref).max()
    assert rel <= 1e-2, rel


def _star_of_copies(n_copies=300, width=31, seed=0):
    """Row 0 plus n_copies rows that each swap one of its columns: node 0 gets
    a few hundred children, so its children list is summed in chunks."""
    rng = np.random.default_rng(seed)
    n = n_copies + 1 + width + 50
    base = np.arange(n_copies + 1, n_copies + 1 + width)
    rows, cols = [], []
    for r in range(n_copies + 1):
        c = base.copy()
        if r > 0:
            c[rng.integers(0, width)] = n_copies + 1 + width + rng.integers(0, 50)
        rows += [r] * len(np.unique(c))
        cols += np.unique(c).tolist()
    return np.array([rows, cols], dtype=np.int32), n


@pytest.mark.parametrize("cols", [40, 256])
def test_adjoint_many_children(cols):
    dev = torch.device("cuda")
    ei, n = _star_of_copies()
    a = _make("ax", ei)
    kids = np.bincount(a.mca_src_idx.cpu().numpy(), minlength=n)
    assert kids.max() > 64, kids.max()
    g = torch.randn(a.num_nodes, cols, device=dev)
    dx = torch.empty_like(g)
    a.adjoint(g, dx)
    ref = _adj_f64("ax", ei, a.num_nodes, g)
    assert np.abs(dx.cpu().numpy() - ref).max() <= 1e-4 * np.abs(ref).max()
    a.plan.check_device()


@pytest.mark.parametrize("graph", ["near_dup", "directed", "chain", "hub"])
def test_transposed_index_sorted_on_device_equals_host_counting_sort(graph):
    """The adjoint's transposed delta matrix is sorted on the GPU (radix sort of
    (column, row) keys); a host counting sort must give the same words."""
    from cbm import _lib

    if graph == "near_dup":
        ei, n = near_dup_graph(4000, seed=3), 4000
    elif graph == "directed":
        n = 3000
        ei = random_graph(n, 6, seed=9, symmetric=False)
    elif graph == "chain":
        ei, n = chain_graph(500)
    else:
        # one column gathered by every row: a long transposed list (chunked)
        n = 2000
        r = np.arange(1, n, dtype=np.int32)
        ei = np.concatenate([np.stack([r, np.zeros_like(r)]), np.stack([np.zeros_like(r), r])], axis=1)
        ei = np.ascontiguousarray(ei[:, np.lexsort((ei[1], ei[0]))])
    a = _make("ax", ei)
    p = a.plan
    assert p._lib.cbm_plan_debug_check_transpose(p._h, None) == _lib.OK
    g = torch.randn(a.num_nodes, 40, device="cuda")
    d1 = torch.empty_like(g)
    d2 = torch.empty_like(g)
    a.adjoint(g, d1)
    a.adjoint(g, d2)
    assert torch.equal(d1, d2)
    ref = _adj_f64("ax", ei, a.num_nodes, g)
    assert np.abs(d1.cpu().numpy() - ref).max() <= 1e-4 * max(1.0, np.abs(ref).max())
    p.check_device()


def test_backward_of_a_self_adjoint_operator_is_its_forward():
    """A symmetric A: cbm4mm and cbm4dad are their own transposes, so autograd's
    backward runs the forward product (bit-identical to matmul on g) and still
    matches the adjoint kernels and FP64; cbm4ad (A D^-1/2) is not, and on a
    directed graph nothing is."""
    from cbm import cbm_mkl_cpp

    dev = torch.device("cuda")
    n = 2500
    ei = near_dup_graph(n, seed=33)
    assert cbm_mkl_cpp.build(ei[0], ei[1], n, 0).symmetric
    for op in ("ax", "dadx", "adx"):
        a = _make(op, ei)
        assert a.self_adjoint == (op != "adx")
        x = torch.randn(n, 24, device=dev, requires_grad=True)
        w = torch.randn(n, 24, device=dev)
        (a.forward(x) * w).sum().backward()
        via_kernels = torch.empty(n, 24, device=dev)
        a.adjoint(w, via_kernels)
        torch.testing.assert_close(x.grad, via_kernels, rtol=1e-5, atol=1e-5)
        if a.self_adjoint:
            fwd = torch.empty(n, 24, device=dev)
            a.matmul(w, fwd)
            assert torch.equal(x.grad, fwd)
        a.plan.check_device()
    directed = random_graph(1500, 8, seed=9, symmetric=False)
    d = _make("ax", directed)
    assert not d.symmetric and not d.self_adjoint
