"""bench.py's measurement helpers on the CPU: the algorithmic byte count and
the sampled FP64 error (checked against the oracle's FP64 product)."""
import numpy as np
import torch

from conftest import near_dup_graph


def test_bytes_alg_counts_each_term():
    import bench

    n, z, e, b, c = 10, 30, 4, 2, 8
    base = 4 * (n + 1) + 4 * z + z * c * 4 + n * c * 4 + e * (8 + 4 * c) + 4 * (b + 1)
    assert bench.bytes_alg(n, z, e, b, c, scaled=False) == base
    assert bench.bytes_alg(n, z, e, b, c) == base + 4 * n
    assert bench.bytes_alg(n, z, e, b, c, sx=2, sy=4, scaled=False) == base - z * c * 2


def test_fp64_sample_error_matches_a_full_fp64_product(oracle_mod):
    import bench

    ei = near_dup_graph(600, seed=3)
    n = int(ei.max()) + 1
    x = torch.randn(n, 16)
    ptr, idx = oracle_mod.csr_from_edges(ei, n)
    d = bench.dinv_f64(ei, n)
    ref = oracle_mod.dense_f64(ptr, idx, n, x.double().numpy(), rs=d, cs=d)
    y = torch.from_numpy(ref.astype(np.float32))
    err = bench.fp64_sample_error(ei, n, x, y, rs=d, cs=d, rows=n)
    assert err["rows_sampled"] == n and err["max_rel"] < 1e-6
    y[5] += 1.0  # one wrong row is seen when every row is sampled
    assert bench.fp64_sample_error(ei, n, x, y, rs=d, cs=d, rows=n)["max_abs"] > 0.5
