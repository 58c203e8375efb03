"""cbm_matmul_noalloc: the product for callers that cannot allocate device memory.

Who needs it: code that runs inside a process whose own allocator already owns
the GPU's memory (a plugin or an inference server that reserves all HBM up
front), a serving loop that must not pay cudaMalloc's implicit device
synchronisation, or an extension point that is only ever handed buffers.  Such
callers cannot build a plan (cbm_plan_create allocates the device layout) nor
allocate the workspace cbm_matmul asks for.  cbm_matmul_noalloc reads the
reference's layout (delta CSR + BFS edge list) from the caller's buffers and
keeps its scratch in a fixed array inside the library.

Checked here through the C ABI against the plan path (cbm_matmul) on the same
inputs, for two calls in a row, at the tolerance the other parity tests use
(rtol 1e-5, atol 1e-6), and bit for bit against the oracle (both sum each row
in entry order and propagate with the reference GPU's rounding).  The
device-side checks are exercised too: a column out of range (CBM_ERR_INDEX), a
node given two parents (CBM_ERR_STRUCTURE) and a chain whose edges are listed
child first, whose bounded wait runs out (CBM_ERR_TIMEOUT, about one second);
after each, the next call is exact again.  Kept in a file of its own,
collected last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import chain_graph, near_dup_graph

pytestmark = pytest.mark.gpu
RTOL, ATOL = 1e-5, 1e-6


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _noalloc(lib, a, x, y, status, mult, col=None, src=None, dst=None):
    crow = a.deltas.crow_indices()
    col = a.deltas.col_indices() if col is None else col
    vals = a.deltas.values()
    src = a.mca_src_idx if src is None else src
    dst = a.mca_dst_idx if dst is None else dst
    n = a.num_nodes
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return lib.cbm_matmul_noalloc(_ptr(crow), _ptr(col), _ptr(vals), n, n, _ptr(src), _ptr(dst), src.numel(),
                                  _ptr(mult), _ptr(x), _ptr(y), x.shape[1], _ptr(status), stream)


def _oracle(a, x, mult):
    from oracle import oracle

    crow = a.deltas.crow_indices().cpu().numpy()
    col = a.deltas.col_indices().cpu().numpy()
    val = a.deltas.values().cpu().numpy()
    br, src, dst = (t.cpu().numpy() for t in (a.mca_offset, a.mca_src_idx, a.mca_dst_idx))
    if mult is None:
        return oracle.spmm_update(crow, col, val, x.cpu().numpy(), br, src, dst)
    return oracle.spmm_fused_update(crow, col, val, x.cpu().numpy(), br, src, dst, mult.cpu().numpy(),
                                    gpu_order=True)


@pytest.mark.parametrize("case", ["dadx-near-dup", "ax-near-dup", "ax-chain"])
def test_noalloc_matches_plan_path_twice(case):
    from cbm import _lib
    from cbm.cbm4dad import cbm4dad
    from cbm.cbm4mm import cbm4mm

    lib = _lib.load()
    dev = torch.device("cuda")
    if case == "ax-chain":
        ei, n = chain_graph(400)
    else:
        n = 3000
        ei = near_dup_graph(n, seed=17, deg=12)
    cls = cbm4dad if case.startswith("dadx") else cbm4mm
    a = cls(torch.from_numpy(ei), torch.ones(ei.shape[1]), alpha=0)
    mult = a.D if case.startswith("dadx") else None
    status = torch.full((1,), -1, dtype=torch.int32, device=dev)
    for call in range(2):
        g = torch.Generator(device=dev).manual_seed(call)
        x = torch.randn(a.num_nodes, 96, device=dev, generator=g)
        y_plan = torch.empty_like(x)
        a.matmul(x, y_plan)  # the existing entry point, cbm_matmul
        y = torch.full_like(x, float("nan"))
        status.fill_(-1)
        assert _noalloc(lib, a, x, y, status, mult) == _lib.OK
        torch.cuda.synchronize()
        assert int(status.item()) == _lib.OK
        torch.testing.assert_close(y, y_plan, rtol=RTOL, atol=ATOL)
        assert np.array_equal(y.cpu().numpy(), _oracle(a, x, mult))


def _check_recovers(lib, a, mult, status):
    """A correct call after a failed one: status OK and bit-exact to the oracle."""
    from cbm import _lib

    x = torch.randn(a.num_nodes, 40, device="cuda")
    y = torch.full_like(x, float("nan"))
    status.fill_(-1)
    assert _noalloc(lib, a, x, y, status, mult) == _lib.OK
    torch.cuda.synchronize()
    assert int(status.item()) == _lib.OK
    assert np.array_equal(y.cpu().numpy(), _oracle(a, x, mult))


def test_noalloc_reports_device_errors_and_recovers():
    from cbm import _lib
    from cbm.cbm4dad import cbm4dad

    lib = _lib.load()
    n = 2000
    ei = near_dup_graph(n, seed=23, deg=10)
    a = cbm4dad(torch.from_numpy(ei), torch.ones(ei.shape[1]), alpha=0)
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    x = torch.randn(n, 40, device="cuda")
    y = torch.empty_like(x)
    # a column index out of range: skipped, reported
    bad_col = a.deltas.col_indices().clone()
    bad_col[7] = n + 3
    assert _noalloc(lib, a, x, y, status, a.D, col=bad_col) == _lib.OK
    torch.cuda.synchronize()
    assert int(status.item()) == _lib.ERR_INDEX
    _check_recovers(lib, a, a.D, status)
    # a node with two parents
    src = torch.cat([a.mca_src_idx, a.mca_src_idx[:1]])
    dst = torch.cat([a.mca_dst_idx, a.mca_dst_idx[-1:]])
    assert _noalloc(lib, a, x, y, status, a.D, src=src, dst=dst) == _lib.OK
    torch.cuda.synchronize()
    assert int(status.item()) == _lib.ERR_STRUCTURE
    _check_recovers(lib, a, a.D, status)


def test_noalloc_wait_runs_out_on_child_first_order_and_recovers():
    """A chain's edges listed deepest first: the first claimed edge waits on a
    parent row that only a later edge of the same claim finishes, so the bounded
    wait (1 s) runs out and reports CBM_ERR_TIMEOUT; the kernel returns and the
    next call is exact."""
    from cbm import _lib
    from cbm.cbm4mm import cbm4mm

    lib = _lib.load()
    ei, n = chain_graph(64)
    a = cbm4mm(torch.from_numpy(ei), torch.ones(ei.shape[1]), alpha=0)
    assert a.mca_src_idx.numel() >= 32
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    x = torch.randn(a.num_nodes, 16, device="cuda")
    y = torch.empty_like(x)
    src = a.mca_src_idx.flip(0).contiguous()
    dst = a.mca_dst_idx.flip(0).contiguous()
    assert _noalloc(lib, a, x, y, status, None, src=src, dst=dst) == _lib.OK
    torch.cuda.synchronize()
    assert int(status.item()) == _lib.ERR_TIMEOUT
    _check_recovers(lib, a, None, status)


def test_noalloc_rejects_rows_beyond_its_scratch():
    from cbm import _lib

    lib = _lib.load()
    too_many = _lib.NOALLOC_MAX_ROWS + 1
    rc = lib.cbm_matmul_noalloc(None, None, None, too_many, too_many, None, None, 0, None, None, None, 8, None, None)
    assert rc == _lib.ERR_TOO_LARGE
    assert "cbm_matmul_noalloc" in _lib.status_string(rc)
