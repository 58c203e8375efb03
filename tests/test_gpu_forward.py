"""GPU parity of the forward products against the oracle (CPU restatement of
the reference's products, cbm/cbm.cu:150-268 and cbm/cbm_extensions.cpp:351-698).

Rows that are not split into chunks are summed in the same order as the
oracle (sequential FMAs over the row's entries) and the propagation uses the
reference's arithmetic, so those results must be bit-identical.  Split rows
are summed chunk by chunk, in another order: there the difference to the
FP64 product and to the oracle is bounded by 1e-5 * |P||Delta||X| + 1e-6,
the magnitude of what was summed (plain rtol fails on cancelling entries).
"""
import numpy as np
import pytest
import torch

from conftest import chain_graph, near_dup_graph, random_graph

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-5, 1e-6


def _dev():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch.device("cuda")


def _make(cls_name, ei, alpha=0):
    from cbm import cbm4ad, cbm4dad, cbm4mm

    cls = {"ax": cbm4mm.cbm4mm, "adx": cbm4ad.cbm4ad, "dadx": cbm4dad.cbm4dad}[cls_name]
    return cls(torch.from_numpy(ei), torch.ones(ei.shape[1]), alpha=alpha)


def _oracle(op, a, x):
    from oracle import oracle

    crow = a.deltas.crow_indices().cpu().numpy()
    col = a.deltas.col_indices().cpu().numpy()
    val = a.deltas.values().cpu().numpy()  # the reference's prepared values
    br = a.mca_offset.cpu().numpy()
    src = a.mca_src_idx.cpu().numpy()
    dst = a.mca_dst_idx.cpu().numpy()
    xn = x.float().cpu().numpy()
    if op == "dadx":
        return oracle.spmm_fused_update(crow, col, val, xn, br, src, dst, a.D.cpu().numpy(), gpu_order=True)
    return oracle.spmm_update(crow, col, val, xn, br, src, dst)


def _f64(op, ei, n, x):
    from oracle import oracle

    ptr, idx = oracle.csr_from_edges(ei, n)
    d = np.diff(ptr).astype(np.float64)
    with np.errstate(divide="ignore"):
        dinv = 1.0 / np.sqrt(d)
    dinv[d == 0] = 0.0  # an empty row's product is 0 (inf * 0 in exact form)
    rs = dinv if op == "dadx" else None
    cs = dinv if op in ("adx", "dadx") else None
    return oracle.dense_f64(ptr, idx, n, x.double().cpu().numpy(), rs=rs, cs=cs)


GRAPHS = {
    "near_dup": lambda: (near_dup_graph(3000, seed=11, deg=14), 3000),
    "random": lambda: (random_graph(2000, 9, seed=4), 2000),
    "community": lambda: (__import__("cbm.synthetic", fromlist=["x"]).workload("community-4096")[0], 4096),
}


@pytest.mark.parametrize("graph", list(GRAPHS))
@pytest.mark.parametrize("op", ["ax", "adx", "dadx"])
@pytest.mark.parametrize("cols", [64, 256])
@pytest.mark.parametrize("variant", ["register", "staged"])
@pytest.mark.parametrize("passes", ["fused", "two"])
def test_forward_bit_exact_vs_oracle(graph, op, cols, variant, passes):
    dev = _dev()
    ei, n = GRAPHS[graph]()
    a = _make(op, ei, alpha=0)
    a.plan.tune(variant=variant, rows_per_claim=5)
    a.plan.set_passes(passes)
    assert a.plan.stat(7) == 0, "no row should be split at these sizes"
    g = torch.Generator(device="cpu").manual_seed(0)
    x = (torch.rand(n, cols, generator=g) * 2 - 1).to(dev)
    y = torch.empty(n, cols, device=dev)
    a.matmul(x, y)
    torch.cuda.synchronize()
    ref = _oracle(op, a, x)
    np.testing.assert_array_equal(y.cpu().numpy(), ref)
    # and close to the exact product
    y64 = _f64(op, ei, n, x)
    err = np.abs(y.cpu().numpy() - y64).max()
    assert err < 1e-4 * max(1.0, np.abs(y64).max())
    a.plan.check_device()


@pytest.mark.parametrize("op", ["ax", "dadx"])
@pytest.mark.parametrize("variant", ["register", "staged", "tma"])
def test_split_rows(op, variant):
    """Force chunking (rows longer than 32 entries) and compare to the oracle."""
    dev = _dev()
    from cbm.synthetic import chung_lu_graph, near_duplicates

    rng = np.random.Generator(np.random.PCG64(3))
    ei = near_duplicates(chung_lu_graph(5000, 2.1, 20.0, rng=rng), 5000, 0.3, 0.1, rng=rng)
    a = _make(op, ei, alpha=0)
    a.plan.tune(chunk_nnz=32, rows_per_claim=2, variant=variant)
    st = a.plan.stats
    assert st["chunks"] > 0 and st["long_rows"] > 0
    x = torch.randn(5000, 128, device=dev)
    y = torch.empty_like(x)
    a.matmul(x, y)
    # chunks are summed separately, so the order differs from the oracle's:
    # bound the difference by the magnitude of what was summed, S = |P||Delta||X|
    ref = _oracle(op, a, x)
    y64 = _f64(op, ei, 5000, x)
    s = _abs_sum(op, a, x)
    out = y.cpu().numpy()
    # a sequential fp32 sum of n terms is within n * 2^-24 * sum|terms| (the
    # oracle's own error); n = longest row + depth
    n_terms = int(np.diff(a.deltas.crow_indices().cpu().numpy()).max()) + st["levels"] + 2
    gamma = max(1e-5, 2.0 * n_terms * 2.0 ** -24)
    over64 = np.abs(out - y64) - (1e-5 * s + 1e-6)
    assert over64.max() <= 0, (over64.max(), np.unravel_index(over64.argmax(), over64.shape))
    over = np.abs(out - ref) - (gamma * s + 1e-6)
    assert over.max() <= 0, (over.max(), np.unravel_index(over.argmax(), over.shape))
    a.plan.check_device()


def _abs_sum(op, a, x):
    """|P| |Delta_op| |X| in fp64: what a product in any summation order adds up."""
    from oracle import oracle

    crow = a.deltas.crow_indices().cpu().numpy()
    col = a.deltas.col_indices().cpu().numpy()
    val = np.abs(a.deltas.values().cpu().numpy()).astype(np.float64)
    xa = np.abs(x.double().cpu().numpy())
    n = crow.size - 1
    s = np.zeros((n, xa.shape[1]))
    rows = np.repeat(np.arange(n), np.diff(crow))
    np.add.at(s, rows, val[:, None] * xa[col])
    src, dst = a.mca_src_idx.cpu().numpy(), a.mca_dst_idx.cpu().numpy()
    ratio = np.ones(src.size)
    if op == "dadx":
        dd = a.D.double().cpu().numpy()
        ratio = dd[dst] / dd[src]
    for u, v, r in zip(src, dst, ratio):
        s[v] += s[u] * r
    return s


@pytest.mark.parametrize("variant", ["register", "staged"])
@pytest.mark.parametrize("passes", ["auto", "fused", "two"])
def test_deep_chain(variant, passes):
    """A 600-deep chain: every row waits on its parent."""
    dev = _dev()
    ei, n = chain_graph(600)
    a = _make("ax", ei)
    a.plan.tune(variant=variant)
    a.plan.set_passes(passes)
    assert a.plan.stats["levels"] == 600
    x = torch.randn(n, 32, device=dev)
    y = torch.empty_like(x)
    a.matmul(x, y)
    np.testing.assert_array_equal(y.cpu().numpy(), _oracle("ax", a, x))
    a.plan.check_device()


@pytest.mark.parametrize("cols", [1, 3, 40, 1100])
def test_column_counts(cols):
    """Scalar path (odd widths), partial teams and the column split beyond 1024."""
    dev = _dev()
    ei = near_dup_graph(1500, seed=2)
    a = _make("dadx", ei)
    x = torch.randn(1500, cols, device=dev)
    y = torch.empty_like(x)
    a.matmul(x, y)
    np.testing.assert_array_equal(y.cpu().numpy(), _oracle("dadx", a, x))


def test_strided_and_misaligned_views():
    dev = _dev()
    ei = near_dup_graph(1200, seed=6)
    a = _make("ax", ei)
    big = torch.randn(1200, 136, device=dev)
    out = torch.zeros(1200, 136, device=dev)
    # leading dimension 136, 64 columns, 16-byte aligned: vector path
    a.matmul(big[:, :64], out[:, :64])
    np.testing.assert_array_equal(out[:, :64].cpu().numpy(), _oracle("ax", a, big[:, :64].contiguous()))
    assert torch.all(out[:, 64:] == 0)
    # offset by one column: scalar path
    a.matmul(big[:, 1:65], out[:, 1:65])
    np.testing.assert_array_equal(out[:, 1:65].cpu().numpy(), _oracle("ax", a, big[:, 1:65].contiguous()))


@pytest.mark.parametrize("ydt", [torch.float32, torch.bfloat16])
@pytest.mark.parametrize("variant", ["register", "staged"])
def test_bf16_inputs(ydt, variant):
    """BF16 X, FP32 accumulation: equal to the fp32 oracle on the same (bf16) values."""
    dev = _dev()
    ei = near_dup_graph(2500, seed=8)
    a = _make("dadx", ei)
    a.plan.tune(variant=variant)
    x = torch.randn(2500, 128, device=dev).to(torch.bfloat16)
    y = torch.empty(2500, 128, device=dev, dtype=ydt)
    a.matmul(x, y)
    ref = torch.from_numpy(_oracle("dadx", a, x))
    assert torch.equal(y.cpu(), ref.to(ydt))


def test_dropin_cusparseCBM_reference_preparation():
    """The reference's own preparation (cbm/cbm4mm.py:26-51, cbm/cbm4dad.py:11-51) fed to cusparseCBM."""
    dev = _dev()
    from cbm import cbm_mkl_cpp
    from cbm.cbm_cusparse import cusparseCBM

    ei = torch.from_numpy(near_dup_graph(2000, seed=3))
    n = int(max(ei[0].max(), ei[1].max())) + 1
    data = cbm_mkl_cpp.init(ei[0], ei[1], torch.ones(ei.shape[1]), n, 0)
    deltas = torch.sparse_coo_tensor(torch.stack([data[0], data[1]]).to(torch.int32), data[2],
                                     (n, n)).coalesce().to_sparse_csr()
    deltas = torch.sparse_csr_tensor(deltas.crow_indices().to(torch.int32), deltas.col_indices().to(torch.int32),
                                     deltas.values().to(torch.float32), deltas.shape).to(dev)
    br, src, dst = (t.to(dtype=torch.int32, device=dev) for t in data[3:])
    ext = cusparseCBM(deltas, br, src, dst, torch.empty(0, device=dev))
    d = torch.zeros(n, 1, device=dev)
    assert ext.matmul_AX_ADX(torch.ones(n, 1, device=dev), d) == 0
    D = (d ** (-1 / 2)).view(-1)
    vals = deltas.values() * D[deltas.col_indices()]
    rows = torch.repeat_interleave(torch.arange(n, device=dev), torch.diff(deltas.crow_indices()))
    vals = vals * D[rows]
    dad = torch.sparse_csr_tensor(deltas.crow_indices(), deltas.col_indices(), vals, deltas.shape)
    ext2 = cusparseCBM(dad, br, src, dst, D)
    x = torch.rand(n, 96, device=dev)
    y = torch.empty_like(x)
    assert ext2.matmul_DAX_DADX(x, y) == 0
    from oracle import oracle

    ref = oracle.spmm_fused_update(dad.crow_indices().cpu().numpy(), dad.col_indices().cpu().numpy(),
                                   vals.cpu().numpy(), x.cpu().numpy(), br.cpu().numpy(), src.cpu().numpy(),
                                   dst.cpu().numpy(), D.cpu().numpy())
    np.testing.assert_array_equal(y.cpu().numpy(), ref)
    with pytest.raises(RuntimeError):
        ext.matmul_DAX_DADX(x, y)


def test_isolated_nodes_dad():
    dev = _dev()
    ei = random_graph(800, 6, seed=1, isolated=50)
    a = _make("dadx", ei)
    assert torch.isinf(a.D).sum() >= 50
    x = torch.randn(800, 64, device=dev)
    y = torch.empty_like(x)
    a.matmul(x, y)
    out = y.cpu().numpy()
    np.testing.assert_array_equal(out, _oracle("dadx", a, x))
    assert np.all(out[200:250] == 0)  # the isolated rows


def test_operand_errors():
    dev = _dev()
    a = _make("ax", near_dup_graph(300, seed=1))
    x = torch.randn(300, 16, device=dev)
    y = torch.empty(300, 16, device=dev)
    with pytest.raises(RuntimeError):
        a.matmul(x.cpu(), y)
    with pytest.raises(RuntimeError):
        a.matmul(x.double(), y)
    with pytest.raises(RuntimeError):
        a.matmul(x[:200], y[:200])
    with pytest.raises(RuntimeError):
        a.matmul(x, torch.empty(300, 8, device=dev))
    with pytest.raises(RuntimeError):
        a.matmul(x, x)  # aliasing
    with pytest.raises(RuntimeError):
        a.matmul(x.to(torch.float32), y.to(torch.bfloat16))  # fp32 -> bf16 is not a supported pair


def test_repeatable_and_graph_capturable():
    dev = _dev()
    a = _make("dadx", near_dup_graph(3000, seed=12))
    x = torch.randn(3000, 64, device=dev)
    y1 = torch.empty_like(x)
    y2 = torch.empty_like(x)
    a.matmul(x, y1)
    a.matmul(x, y2)
    assert torch.equal(y1, y2)
    # capture in a CUDA graph and replay on new inputs
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        a.matmul(x, y2)
    torch.cuda.current_stream().wait_stream(s)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        a.matmul(x, y2)
    for seed in range(3):
        x.copy_(torch.randn(3000, 64, device=dev, generator=torch.Generator(device=dev).manual_seed(seed)))
        graph.replay()
        a.matmul(x, y1)
        torch.cuda.synchronize()
        assert torch.equal(y1, y2)
    a.plan.check_device()


@pytest.mark.parametrize("passes", ["fused", "two"])
def test_bounded_wait_times_out_and_recovers(passes):
    """A row made to wait on a flag that nothing sets: the kernel returns, the
    status says timeout, and the plan keeps working.  Fused: a level-0 item
    given a leaf as its parent.  Two passes: the deepest item given a leaf
    below level 0 as its parent (the propagation pass waits on such parents)."""
    dev = _dev()
    from cbm import _lib

    n = 500
    a = _make("ax", near_dup_graph(n, seed=4))
    p = a.plan
    p.set_passes(passes)
    par = np.asarray(a.parent)
    depth = np.zeros(n, np.int64)
    for v in range(n):
        u = v
        while par[u] != n:
            u = par[u]
            depth[v] += 1
    order = np.argsort(depth, kind="stable")  # the plan's item order: by level, stable by node id
    has_child = set(a.mca_src_idx.cpu().tolist())
    if passes == "fused":
        item = 0
        leaf = next(v for v in range(n) if v not in has_child)
    else:
        item = n - 1
        leaf = next(int(v) for v in order[::-1] if depth[v] > 0 and int(v) not in has_child and v != order[item])
    p.set_timeout(5_000_000)  # 5 ms
    rc = p._lib.cbm_plan_debug_set_parent(p._h, item, leaf, None)
    assert rc == 0
    x = torch.randn(n, 32, device=dev)
    y = torch.empty_like(x)
    a.matmul(x, y)
    st, info = p.error()
    assert st == _lib.ERR_TIMEOUT
    # restore the item's own parent
    own = int(par[order[item]])
    assert p._lib.cbm_plan_debug_set_parent(p._h, item, -1 if own == n else own, None) == 0
    p.set_timeout(1_000_000_000)
    a.matmul(x, y)
    assert p.error()[0] == _lib.OK
    np.testing.assert_array_equal(y.cpu().numpy(), _oracle("ax", a, x))


@pytest.mark.parametrize("team", [8, 16, 32])
@pytest.mark.parametrize("cols,dtype", [(256, torch.float32), (64, torch.float32), (128, torch.bfloat16),
                                        (512, torch.float32)])
@pytest.mark.parametrize("hot_rows", [65536, 0])
def test_staged_team_shapes(team, cols, dtype, hot_rows):
    """Every team size of the staged kernel (several row streams per warp stepping
    together) gives the oracle's result bit for bit on unsplit rows, with L2
    policies per entry (a hot set) and without (hot_rows 0)."""
    dev = _dev()
    ei = near_dup_graph(3000, seed=23, deg=14)
    a = _make("dadx", ei)
    a.plan.tune(variant="staged", team=team, rows_per_claim=3, hot_rows=hot_rows)
    x = torch.randn(3000, cols, device=dev).to(dtype)
    y = torch.empty(3000, cols, device=dev)
    a.matmul(x, y)
    np.testing.assert_array_equal(y.cpu().numpy(), _oracle("dadx", a, x))
    a.plan.check_device()


@pytest.mark.parametrize("cols,dtype,op", [(128, torch.bfloat16, "adx"), (64, torch.float32, "dadx"),
                                           (256, torch.float32, "dadx"), (128, torch.float32, "ax"),
                                           (64, torch.bfloat16, "ax"), (256, torch.bfloat16, "dadx")])
def test_tma_gather_variant_bit_exact(cols, dtype, op):
    """The TMA variant (rows gathered four at a time by tile::gather4) sums in the
    same order as the oracle: bit-identical results, split rows included."""
    dev = _dev()
    ei = near_dup_graph(3000, seed=41, deg=14)
    a = _make(op, ei)
    a.plan.tune(variant="tma", rows_per_claim=3)
    assert a.plan.stats["chunks"] == 0
    x = torch.randn(3000, cols, device=dev).to(dtype)
    y = torch.empty(3000, cols, device=dev)
    for _ in range(2):
        a.matmul(x, y)
        a.plan.check_device()
        np.testing.assert_array_equal(y.cpu().numpy(), _oracle(op, a, x))


@pytest.mark.parametrize("op", ["ax", "adx", "dadx"])
@pytest.mark.parametrize("cols", [40, 128])
def test_two_pass_equals_fused_on_a_deep_tree(op, cols):
    """On a tree where most rows hang below level 0 (where AUTO takes two
    passes), the two-pass product equals the fused one and the oracle bit for
    bit, for BF16 X too (FP32 Y)."""
    dev = _dev()
    ei = near_dup_graph(6000, seed=41, frac=0.8, flip=0.05, deg=10)
    a = _make(op, ei, alpha=0)
    st = a.plan.stats
    assert st["levels"] >= 3 and st["chunks"] == 0
    for xdt in (torch.float32, torch.bfloat16):
        x = torch.randn(6000, cols, device=dev).to(xdt)
        ys = {}
        for passes in ("fused", "two", "auto"):
            a.plan.set_passes(passes)
            y = torch.full((6000, cols), float("nan"), device=dev)
            a.matmul(x, y)
            ys[passes] = y.cpu().numpy()
        assert np.array_equal(ys["two"], ys["fused"])
        assert np.array_equal(ys["auto"], ys["fused"])
        np.testing.assert_array_equal(ys["two"], _oracle(op, a, x.float()))
    a.plan.check_device()


@pytest.mark.parametrize("variant", ["staged", "register"])
@pytest.mark.parametrize("dtype", [torch.bfloat16, torch.float32])
def test_row_offsets_past_32_bits(variant, dtype):
    """An X view whose row offsets pass 2^32 elements (leading dimension
    2,100,000 over 2,100 rows) takes the kernels' 64-bit row addressing; the
    product equals, bit for bit, the one on a compact copy of X (32-bit row
    offsets) and the oracle's."""
    dev = _dev()
    n, cols, ld = 2100, 128, 2_100_000
    assert (n - 1) * ld + cols > 2 ** 32
    a = _make("ax", near_dup_graph(n, seed=12))
    a.plan.tune(variant=variant)
    # 8.8 GB (BF16) or 17.6 GB (FP32); only the view's n rows are written
    buf = torch.empty((n - 1) * ld + cols, dtype=dtype, device=dev)
    xv = buf.as_strided((n, cols), (ld, 1))
    xc = torch.randn(n, cols, device=dev).to(dtype)
    xv.copy_(xc)
    y_wide = torch.empty(n, cols, device=dev)
    y_compact = torch.empty_like(y_wide)
    a.matmul(xv, y_wide)
    a.matmul(xc, y_compact)
    torch.cuda.synchronize()
    del xv, buf
    torch.cuda.empty_cache()
    assert torch.equal(y_wide, y_compact)
    np.testing.assert_array_equal(y_compact.cpu().numpy(), _oracle("ax", a, xc.float()))
    a.plan.check_device()
