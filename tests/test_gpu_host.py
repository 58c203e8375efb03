"""Products with host-resident operands (cbm_matmul_host): column slabs copied
in, multiplied and copied out on overlapping streams must give exactly the
device product, for every slab width, dtype pair and pinned or pageable
host memory."""
import numpy as np
import pytest
import torch

from conftest import near_dup_graph

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def op_dad():
    from cbm.cbm4dad import cbm4dad

    ei = near_dup_graph(5000, seed=29, deg=16)
    return cbm4dad(torch.from_numpy(ei), torch.ones(ei.shape[1]), alpha=0)


@pytest.mark.parametrize("cols,slab", [(256, 64), (256, 0), (256, 100), (96, 32), (70, 16), (8, 3)])
@pytest.mark.parametrize("dt", [(torch.float32, torch.float32), (torch.bfloat16, torch.float32)])
@pytest.mark.parametrize("pinned", [True, False])
def test_host_product_equals_device_product(op_dad, cols, slab, dt, pinned):
    xdt, ydt = dt
    n = op_dad.num_nodes
    g = torch.Generator().manual_seed(cols + slab)
    xh = torch.randn(n, cols, generator=g).to(xdt)
    yh = torch.full((n, cols), float("nan"), dtype=ydt)
    if pinned:
        xh, yh = xh.pin_memory(), yh.pin_memory()
    op_dad.matmul_host(xh, yh, slab_cols=slab)
    torch.cuda.current_stream().synchronize()
    xd = xh.cuda()
    yd = torch.empty(n, cols, dtype=ydt, device="cuda")
    op_dad.matmul(xd, yd)
    np.testing.assert_array_equal(yh.float().numpy(), yd.float().cpu().numpy())
    op_dad.plan.check_device()


def test_host_product_twice_and_errors(op_dad):
    n = op_dad.num_nodes
    xh = torch.randn(n, 64).pin_memory()
    yh = torch.empty(n, 64).pin_memory()
    ref = torch.empty(n, 64, device="cuda")
    for _ in range(2):
        xh.normal_()
        op_dad.matmul_host(xh, yh, slab_cols=16)
        op_dad.matmul(xh.cuda(), ref)
        torch.cuda.synchronize()
        assert torch.equal(yh, ref.cpu())
    with pytest.raises(RuntimeError):
        op_dad.matmul_host(xh.cuda(), yh)
    with pytest.raises(RuntimeError):
        op_dad.matmul_host(xh, torch.empty(n, 32))


@pytest.mark.parametrize("slab", [64, 0, 48])
def test_back_to_back_calls_with_overlap(op_dad, slab):
    """overlap_calls: a call's copy-in runs under the previous call's copy-out.
    Three calls in a row on different inputs and outputs, queued without a
    synchronisation between them, each equal to the device product; then a
    call without overlap after them."""
    n = op_dad.num_nodes
    g = torch.Generator().manual_seed(slab)
    xs = [torch.randn(n, 192, generator=g).pin_memory() for _ in range(3)]
    ys = [torch.full((n, 192), float("nan")).pin_memory() for _ in range(3)]
    for x, y in zip(xs, ys):
        op_dad.matmul_host(x, y, slab_cols=slab, overlap_calls=True)
    last = torch.full((n, 192), float("nan")).pin_memory()
    op_dad.matmul_host(xs[0], last, slab_cols=slab)
    torch.cuda.current_stream().synchronize()
    ref = torch.empty(n, 192, device="cuda")
    for x, y in zip(xs, ys):
        op_dad.matmul(x.cuda(), ref)
        assert torch.equal(y, ref.cpu())
    op_dad.matmul(xs[0].cuda(), ref)
    assert torch.equal(last, ref.cpu())
    op_dad.plan.check_device()


@pytest.mark.parametrize("slab", [64, 96])
def test_overlapped_calls_released_before_copy_out(op_dad, slab):
    """With overlap_calls the current stream waits only for the products: the
    copy-outs finish after host_wait().  Four calls with the same slab layout
    (ordered slab by slab), then one with another slab width (ordered against
    the whole previous call), each equal to the device product."""
    n = op_dad.num_nodes
    g = torch.Generator().manual_seed(100 + slab)
    xs = [torch.randn(n, 192, generator=g).pin_memory() for _ in range(5)]
    ys = [torch.full((n, 192), float("nan")).pin_memory() for _ in range(5)]
    for i, (x, y) in enumerate(zip(xs, ys)):
        op_dad.matmul_host(x, y, slab_cols=slab if i < 4 else 128, overlap_calls=True)
    op_dad.host_wait()
    torch.cuda.current_stream().synchronize()
    ref = torch.empty(n, 192, device="cuda")
    for x, y in zip(xs, ys):
        op_dad.matmul(x.cuda(), ref)
        assert torch.equal(y, ref.cpu())
    op_dad.plan.check_device()
