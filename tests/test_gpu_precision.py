"""Precision form: X stored in BF16, FP32 accumulation, FP32 output; error
against the FP64 oracle stated two ways:

* product error: FP64 product of the same BF16 values (what the kernel adds);
* end-to-end error: FP64 product of the FP32 values before BF16 rounding
  (storage rounding included).

Relative error = ||ours - ref|| / ||ref|| (Frobenius) and max |ours - ref| /
max |ref|.  Default size: 300,000 nodes of the same law as the 2.4M-node
workload; CBM_FULL_WORKLOADS=1 runs the full 2,400,000-node graph.
"""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _errors(out, ref):
    return {"rel_fro": float(np.linalg.norm(out - ref) / np.linalg.norm(ref)),
            "rel_max": float(np.abs(out - ref).max() / np.abs(ref).max())}


def test_precision_form_error_vs_fp64():
    from cbm import synthetic
    from cbm.cbm4ad import cbm4ad
    from oracle import oracle

    if os.environ.get("CBM_FULL_WORKLOADS") == "1":
        ei, n, spec = synthetic.workload("powerlaw-2.4m")
        alpha = spec["alpha"]
    else:
        n = 300_000
        ei = synthetic._w_powerlaw(n, 2.3, 50.0, 0.40, 0.05, 2)
        alpha = 16
    a = cbm4ad(torch.from_numpy(ei), torch.ones(ei.shape[1]), alpha=alpha)
    g = torch.Generator(device="cuda").manual_seed(2)
    x32 = torch.randn(a.num_nodes, 128, device="cuda", generator=g)
    x = x32.to(torch.bfloat16)
    y = torch.empty(a.num_nodes, 128, device="cuda")
    a.matmul(x, y)
    ptr, idx = oracle.csr_from_edges(ei, a.num_nodes)
    deg = np.diff(ptr).astype(np.float64)
    with np.errstate(divide="ignore"):
        dinv = 1.0 / np.sqrt(deg)
    dinv[deg == 0] = 0.0
    out = y.double().cpu().numpy()
    product = _errors(out, oracle.dense_f64(ptr, idx, a.num_nodes, x.double().cpu().numpy(), cs=dinv))
    end_to_end = _errors(out, oracle.dense_f64(ptr, idx, a.num_nodes, x32.double().cpu().numpy(), cs=dinv))
    print(f"precision form N={a.num_nodes}: product error {product}, end-to-end error {end_to_end}")
    assert product["rel_fro"] <= 1e-5
    assert end_to_end["rel_fro"] <= 1e-2
    a.plan.check_device()
