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


def test_clock_record_from_nvml_samples():
    """The clock record taken through NVML: median and minimum SM clock, and
    the union of the clock-event reasons seen, by nvidia-smi's names."""
    import bench

    c = bench.Clocks(0)
    c.thread = object()  # as if the sampling thread had run
    c.max_mhz = 1965.0
    c.rows = [(1965.0, 600.0, 0), (1965.0, 610.0, 0x4), (1905.0, 620.0, 0x0)]
    s = c.summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_min_mhz"] == 1905.0 and s["sm_max_mhz"] == 1965.0
    assert s["samples"] == 3 and s["reasons"] == ["sw_power_cap"]
    c.rows.append((1200.0, 650.0, 0x8 | 0x40))
    assert c.summary()["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_power_cap"]


def test_clock_record_from_nvidia_smi_lines():
    """The fallback record parsed from nvidia-smi's CSV lines: idle samples
    (under 200 W) are left out of the median once loaded ones exist."""
    import bench

    c = bench.Clocks(0)
    c.out = "\n".join([
        "0, 345, 1965, 120.5, 0x0, Not Active, Not Active, Not Active, Not Active",
        "0, 1965, 1965, 700.1, 0x4, Not Active, Not Active, Not Active, Active",
        "0, 1950, 1965, 710.0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ])
    s = c.summary()
    assert s["sm_mhz"] == (1965.0 + 1950.0) / 2 and s["sm_max_mhz"] == 1965.0
    assert s["samples"] == 3 and s["reasons"] == ["sw_power_cap"]


def test_roofline_fractions():
    """Rates are bytes over the launch time against the measured peak."""
    import bench

    peak, _ = bench.peaks()
    r = bench.roofline(2e9, 1e9, 1.0, traffic=1.5e9)
    assert abs(r["achieved"] - 2000.0) < 1e-6 and abs(r["frac"] - 2000.0 / peak) < 1e-9
    assert abs(r["compulsory_achieved"] - 1000.0) < 1e-6 and abs(r["dram_achieved"] - 1500.0) < 1e-6
    assert r["bytes_alg_per_launch"] == 2_000_000_000
