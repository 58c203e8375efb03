"""Golden vectors: the reference's own GPU products on small seeded graphs
(tests/golden/reference_products.npz, made by tests/golden/make_golden.py
with the reference's cbm/cbm.cu and cbm/csr.cu compiled from source).

CPU checks pin the oracle: its fp32 restatements of matmul_AX_ADX and
matmul_DAX_DADX (cbm/cbm.cu:150-268) and its FP64 product over A reproduce
the reference's outputs within the reference's own parity rule (rtol 1e-5,
benchmark/compare_matmul_cuda.py:58-59; atol 1e-6 for entries near zero).
The constructor's output for each case is stored too, and is checked bit for
bit (against this library's constructor and the oracle's emission rules).
The GPU check runs this library's products on the stored structure.
"""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_products.npz")
RTOL, ATOL = 1e-5, 1e-6


def _cases():
    data = np.load(GOLDEN)
    names = sorted({k.split("/")[0] for k in data.files})
    return {name: {k.split("/", 1)[1]: data[k] for k in data.files if k.startswith(name + "/")} for name in names}


CASES = _cases()


@pytest.fixture(params=sorted(CASES))
def case(request):
    return request.param, CASES[request.param]


def test_fixture_covers_the_forms():
    assert len(CASES) >= 5
    assert sum("y_dadx" in c for c in CASES.values()) >= 4
    assert any(int(c["alpha"]) > 0 for c in CASES.values())
    assert any(np.any(np.diff(c["crow"]) == 0) for c in CASES.values())  # empty delta rows


def test_oracle_products_match_reference(case, oracle_mod):
    name, c = case
    o = oracle_mod
    args = (c["branches"], c["src"], c["dst"])
    np.testing.assert_allclose(o.spmm_update(c["crow"], c["col"], c["sign"], c["x"], *args), c["y_ax"],
                               rtol=RTOL, atol=ATOL, err_msg=name)
    ptr, idx = o.csr_from_edges(c["ei"], int(c["n"]))
    a_x = o.dense_f64(ptr, idx, int(c["n"]), c["x"])
    np.testing.assert_allclose(a_x, c["y_csr"], rtol=RTOL, atol=ATOL, err_msg=name)
    # the reference's own validation: CBM product == CSR product
    np.testing.assert_allclose(c["y_ax"], c["y_csr"], rtol=RTOL, atol=ATOL, err_msg=name)
    if "y_dadx" not in c:
        return
    np.testing.assert_allclose(o.spmm_update(c["crow"], c["col"], c["val_ad"], c["x"], *args), c["y_adx"],
                               rtol=RTOL, atol=ATOL, err_msg=name)
    np.testing.assert_allclose(o.spmm_fused_update(c["crow"], c["col"], c["val_dad"], c["x"], *args, c["D"]),
                               c["y_dadx"], rtol=RTOL, atol=ATOL, err_msg=name)
    # D = d^-1/2 with d the exact row degree (inf for empty rows)
    deg = np.diff(ptr)
    with np.errstate(divide="ignore"):
        want = (1.0 / np.sqrt(deg.astype(np.float64))).astype(np.float32)
    np.testing.assert_allclose(c["D"], want, rtol=2e-7)
    # FP64 forms over A
    dinv = np.where(deg > 0, want.astype(np.float64), 0.0)
    np.testing.assert_allclose(o.dense_f64(ptr, idx, int(c["n"]), c["x"], cs=dinv), c["y_adx"], rtol=RTOL,
                               atol=ATOL, err_msg=name)
    np.testing.assert_allclose(o.dense_f64(ptr, idx, int(c["n"]), c["x"], rs=dinv, cs=dinv), c["y_dadx"],
                               rtol=RTOL, atol=ATOL, err_msg=name)


def test_constructor_reproduces_stored_structure(case):
    from cbm import cbm_mkl_cpp

    name, c = case
    ei = c["ei"]
    s = cbm_mkl_cpp.build(np.ascontiguousarray(ei[0]), np.ascontiguousarray(ei[1]), int(c["n"]), int(c["alpha"]))
    for field, key in (("csr_ptr", "crow"), ("csr_col", "col"), ("csr_val", "sign"), ("branches", "branches"),
                       ("src", "src"), ("dst", "dst")):
        np.testing.assert_array_equal(getattr(s, field), c[key], err_msg=f"{name}: {field}")


def test_oracle_emission_reproduces_stored_structure(case, oracle_mod):
    name, c = case
    n = int(c["n"])
    parent = np.full(n, n, np.int32)
    parent[c["dst"]] = c["src"]
    (dr, dc, dv, br, s, d), _ = oracle_mod.reference_structure(c["ei"], n, int(c["alpha"]), parent)
    # the emission is COO in BFS order; cbm4mm coalesces it to CSR (cbm/cbm4mm.py:26-32)
    order = np.lexsort((dc, dr))
    dr, dc, dv = dr[order], dc[order], dv[order]
    crow = np.zeros(n + 1, np.int64)
    np.add.at(crow, dr.astype(np.int64) + 1, 1)
    np.testing.assert_array_equal(np.cumsum(crow), c["crow"], err_msg=name)
    np.testing.assert_array_equal(dc, c["col"], err_msg=name)
    np.testing.assert_array_equal(dv, c["sign"], err_msg=name)
    np.testing.assert_array_equal(br, c["branches"], err_msg=name)
    np.testing.assert_array_equal(s, c["src"], err_msg=name)
    np.testing.assert_array_equal(d, c["dst"], err_msg=name)


@pytest.mark.gpu
def test_gpu_products_match_reference(case):
    import torch

    from cbm.plan import Plan

    name, c = case
    n = int(c["n"])
    plan = Plan(c["crow"], c["col"], c["sign"], n, n, c["branches"], c["src"], c["dst"], host=True)
    x = torch.from_numpy(c["x"]).cuda()
    y = torch.empty_like(x)
    plan.matmul("ax", x, y)
    torch.testing.assert_close(y.cpu(), torch.from_numpy(c["y_ax"]), rtol=RTOL, atol=ATOL)
    if "y_dadx" in c:
        plan.set_multipliers(torch.from_numpy(c["D"]).cuda())
        for op, key in (("adx", "y_adx"), ("dadx", "y_dadx")):
            plan.matmul(op, x, y)
            torch.testing.assert_close(y.cpu(), torch.from_numpy(c[key]), rtol=RTOL, atol=ATOL)
    plan.check_device()
