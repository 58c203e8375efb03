"""Benchmark: CBM D^-1/2 A D^-1/2 X throughput (GB/s of algorithmic bytes) on B200,
and the GCN fwd+bwd time in BF16 against plain FP32.

Workload (default): the 1,000,000-node power-law graph (Chung-Lu exponent 2.1,
mean degree 20, 30% near-duplicate rows with 10% flips, symmetrised, seed 1),
CBM built with alpha = 8, X 1e6 x 256 fp32 N(0,1); one step = one
D^-1/2 A D^-1/2 X product (cbm4dad.matmul).  X and Y (1.02 GB each) exceed
the 126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

The line also carries "gcn": a 2-layer GCN (128 -> 256 -> 40) on the
170,000-node power-law graph (exponent 2.1, mean degree 14, 25% near-duplicate
rows, seed 3), forward + backward ms per step with BF16 activations and with
plain FP32, and their ratio (rank 0 only).

At N = 1 the line also carries the other forms, each measured on the device
with CUDA events after its own warm-up, outside the headline's timed region:
"precision" (A D^-1/2 X on the 2.4M-node workload, X stored BF16), "batch"
(the 512-graph workload in one launch replayed from a CUDA graph), "small"
(A.X on the 4,096-node community graph: launch latency, eager and from a CUDA
graph) and "direct" (the reference's operator s_spmm_fused_update_csr_int32
through its own signature on CUDA tensors, on the headline's structure), with
error against FP64 on sampled rows.

N > 1 runs under torchrun, one rank per GPU: each rank owns a 256-column shard
of X and Y (column sharding needs no collective; weak scaling).  Rank 0
prints one JSON line.  ``--impl reference`` times the reference's CPU product
path (MKL CSR SpMM + OpenMP branch-serial fused update,
s_spmm_fused_update_csr_int32, cbm/cbm_extensions.cpp:593-698), compiled from
its source into oracle/_ref/ (else the oracle's restatement of it), on all
host threads; its line also carries "reference_gpu", the reference's own GPU
products (cusparseCBM, compiled from cbm/cbm.cu) on the headline workload and
on the 4,096-node graph, timed with CUDA events on the same box.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np
import torch

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "cbm-gpu_b200"))

WORKLOAD = "powerlaw-1m"
CACHE = os.path.join(REPO, "_cache")  # generated graphs and constructed CBM structures
COLS = 256
HBM_FALLBACK_GBS = 6650.0


def peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def bytes_alg(n, z, e, b, cols, sx=4, sy=4, scaled=True):
    """Algorithmic bytes of one product: row pointers + column indices, one X-row
    gather per delta entry, Y written once, per tree edge its ids and one fp32
    parent-row read, branch offsets, and the D^-1/2 vector."""
    return (4 * (n + 1) + 4 * z + z * cols * sx + n * cols * sy + e * (8 + 4 * cols) + 4 * (b + 1)
            + (4 * n if scaled else 0))


def bytes_compulsory(n, z, e, b, cols, sx=4, sy=4, scaled=True):
    """Bytes any implementation of one product must move: X read once, Y
    written once, the delta matrix (row pointers, column indices; signs free),
    the tree (ids per edge, branch offsets) and D^-1/2.  X-row gathers that
    miss L2 are re-reads on top of these."""
    return (n * cols * sx + n * cols * sy + 4 * (n + 1) + 4 * z + 8 * e + 4 * (b + 1) + (4 * n if scaled else 0))


def roofline(b_alg, b_min, ms, traffic=None):
    """Roofline record of one launch of ms milliseconds against the measured
    HBM copy peak: the algorithmic (gather) rate, the compulsory-byte rate and,
    given the DRAM bytes of an ncu capture, the DRAM rate."""
    peak, kind = peaks()
    t = ms * 1e-3
    r = {"bound": "hbm", "achieved": b_alg / t / 1e9, "peak": peak, "unit": "GB/s", "frac": b_alg / t / 1e9 / peak,
         "peak_kind": kind, "bytes_alg_per_launch": int(b_alg), "bytes_compulsory_per_launch": int(b_min),
         "compulsory_achieved": b_min / t / 1e9, "frac_compulsory": b_min / t / 1e9 / peak, "traffic": traffic}
    if traffic:
        r["dram_achieved"] = traffic / t / 1e9
        r["dram_frac"] = traffic / t / 1e9 / peak
    return r


def load_graph(rank, world):
    """Edge list of the workload, generated once by rank 0 into a file cache that
    every rank reads after a barrier."""
    from cbm import synthetic
    from cbm.shard import build_once

    cache = os.path.join(REPO, "_cache")
    os.makedirs(cache, exist_ok=True)

    def make(path):
        ei, n, _ = synthetic.workload(WORKLOAD)
        with open(path, "wb") as f:
            np.savez(f, ei=ei, n=n)

    d = np.load(build_once(os.path.join(cache, f"{WORKLOAD}.npz"), make, rank))
    return d["ei"], int(d["n"]), synthetic.WORKLOADS[WORKLOAD]


def fp64_sample_error(ei, n, x, y, rs=None, cs=None, rows=4096, seed=0):
    """Max-abs and relative error of y = rs o (A (cs o x)) on a sample of rows
    against FP64 sums over the original A (the edge list, not the CBM form)."""
    r = np.asarray(ei[0])
    c = np.asarray(ei[1])
    ptr = np.zeros(n + 1, dtype=np.int64)
    ptr[1:] = np.cumsum(np.bincount(r, minlength=n))
    order = np.argsort(r, kind="stable") if np.any(np.diff(r) < 0) else None
    cols = c[order] if order is not None else c
    pick = np.sort(np.random.default_rng(seed).choice(n, size=min(rows, n), replace=False))
    lens = ptr[pick + 1] - ptr[pick]
    nb = np.concatenate([cols[ptr[v]:ptr[v + 1]] for v in pick]).astype(np.int64)
    xs = x[torch.from_numpy(nb).to(x.device)].double().cpu().numpy()
    if cs is not None:
        xs *= cs[nb][:, None]
    starts = np.concatenate([[0], np.cumsum(lens)[:-1]])
    ref = np.zeros((pick.size, xs.shape[1]))
    has = lens > 0
    ref[has] = np.add.reduceat(xs, starts[has], axis=0)
    if rs is not None:
        ref *= rs[pick][:, None]
    out = y[torch.from_numpy(pick).to(y.device)].double().cpu().numpy()
    diff = np.abs(out - ref)
    return {"rows_sampled": int(pick.size), "max_abs": float(diff.max()),
            "max_rel": float(diff.max() / max(np.abs(ref).max(), 1e-300)),
            "rel_fro": float(np.linalg.norm(out - ref) / max(np.linalg.norm(ref), 1e-300))}


def dinv_f64(ei, n):
    deg = np.bincount(np.asarray(ei[0]), minlength=n).astype(np.float64)
    with np.errstate(divide="ignore"):
        d = 1.0 / np.sqrt(deg)
    d[deg == 0] = 0.0
    return d


class Clocks:
    """SM clock, power and clock-event reasons sampled DURING the timed region:
    through NVML every 2 ms from a thread (nvidia_ml_py), else nvidia-smi
    every 200 ms.  Read-only: no clock or other setting is changed."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits and their nvidia-smi names
    REASONS = ((0x8, "hw_slowdown"), (0x40, "hw_thermal_slowdown"), (0x20, "sw_thermal_slowdown"),
               (0x4, "sw_power_cap"), (0x80, "hw_power_brake_slowdown"))

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.thread = None
        self.rows = []
        self.out = ""

    def _nvml(self):
        import pynvml

        pynvml.nvmlInit()
        try:
            u = str(torch.cuda.get_device_properties(self.index).uuid)
            h = pynvml.nvmlDeviceGetHandleByUUID((u if u.startswith("GPU-") else "GPU-" + u).encode())
        except Exception:
            ids = [v.strip() for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
            idx = int(ids[self.index]) if len(ids) > self.index and ids[self.index].isdigit() else self.index
            h = pynvml.nvmlDeviceGetHandleByIndex(idx)
        return pynvml, h

    def __enter__(self):
        try:
            nv, h = self._nvml()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.stop = threading.Event()

            def loop():
                while not self.stop.is_set():
                    try:
                        self.rows.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                          nv.nvmlDeviceGetPowerUsage(h) / 1000.0,
                                          int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))))
                    except Exception:
                        return
                    self.stop.wait(0.002)

            self.thread = threading.Thread(target=loop, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=5)
            return
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.thread is not None:
            if not self.rows:
                return None
            bits = 0
            for r in self.rows:
                bits |= r[2]
            return {"sm_mhz": statistics.median(r[0] for r in self.rows), "sm_max_mhz": self.max_mhz,
                    "sm_min_mhz": min(r[0] for r in self.rows), "power_w_median": statistics.median(r[1] for r in self.rows),
                    "samples": len(self.rows), "source": "NVML every 2 ms inside the timed region",
                    "reasons": sorted(name for bit, name in self.REASONS if bits & bit)}
        rows = []
        for line in (self.out or "").splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), float(parts[3]), parts[5:9]))
            except ValueError:
                continue
        if not rows:
            return None
        loaded = [r for r in rows if r[2] > 200.0] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in loaded for i, v in enumerate(r[3]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in loaded), "sm_max_mhz": max(r[1] for r in rows),
                "samples": len(rows), "source": "nvidia-smi every 200 ms", "reasons": reasons}


def traffic_from_profile():
    """DRAM bytes per launch of the product kernel from the committed ncu
    summary, and where they come from (the summary's file and the commit it
    was captured at)."""
    name = "fwd_stream_kernel_powerlaw-1m.md"
    path = os.path.join(REPO, "profiles", name)
    traffic, commit = None, None
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                traffic = float(line.split(":", 1)[1].split()[0])
            if line.startswith("commit:"):
                commit = line.split(":", 1)[1].strip().split()[0]
    except OSError:
        pass
    return traffic, {"profile": f"profiles/{name}", "commit": commit}


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_cpu_product():
    """(run, kind, what): the reference's own CPU product
    s_spmm_fused_update_csr_int32 (cbm/cbm_extensions.cpp:593-698: MKL
    mkl_sparse_s_mm, then the OpenMP branch-parallel fused update), compiled
    from its source into oracle/_ref/ by oracle/build_ref.py; where that module
    is absent, the oracle's restatement of it (same arithmetic, plain loops).
    run(crow, col, val, x, branches, src, dst, mult) computes one product on all
    host threads."""
    import torch as _t

    from oracle import build_ref, oracle

    mod = build_ref.load(build_ref.CPU_MODULE)
    if mod is not None:
        cache = {}

        def run(crow, col, val, x, br, src, dst, mult):
            key = id(crow), id(x)
            if key not in cache:
                cache.clear()
                ct = _t.from_numpy(np.ascontiguousarray(crow, dtype=np.int32))
                cache[key] = ([ct[:-1].clone(), ct[1:].clone()] +
                              [_t.from_numpy(np.ascontiguousarray(a, dtype=d)) for a, d in
                               ((col, np.int32), (val, np.float32), (x, np.float32), (br, np.int32),
                                (src, np.int32), (dst, np.int32), (mult, np.float32))] +
                              [_t.empty(x.shape, dtype=_t.float32)])
            a = cache[key]
            mod.s_spmm_fused_update_csr_int32(*a)
            return a[-1]

        return run, "reference", "the reference's s_spmm_fused_update_csr_int32 (MKL + OpenMP), built from its source"

    def run(crow, col, val, x, br, src, dst, mult):
        return oracle.spmm_fused_update(crow, col, val, x, br, src, dst, mult, gpu_order=False, parallel=True)

    return run, "port", "the oracle's restatement of s_spmm_fused_update_csr_int32 (OpenMP)"


def cpu_baseline(a, x_np, b_alg, budget_s=15.0):
    """The reference's CPU product path on all host threads, on the same workload."""
    crow = a.deltas.crow_indices().cpu().numpy()
    col = a.deltas.col_indices().cpu().numpy()
    val = a.deltas.values().cpu().numpy()
    br, src, dst = (t.cpu().numpy() for t in (a.mca_offset, a.mca_src_idx, a.mca_dst_idx))
    mult = a.D.cpu().numpy()
    run, kind, what = reference_cpu_product()
    run(crow, col, val, x_np, br, src, dst, mult)  # warm-up (first-touch, MKL set-up)
    times = []
    t_end = time.perf_counter() + budget_s
    while not times or time.perf_counter() < t_end:
        t0 = time.perf_counter()
        run(crow, col, val, x_np, br, src, dst, mult)
        times.append(time.perf_counter() - t0)
        if len(times) >= 10:
            break
    t = statistics.median(times)
    return {"value": b_alg / t / 1e9, "unit": "GB/s", "cores": host_threads(), "kind": kind,
            "ms_per_product": t * 1e3,
            "sample": f"{len(times)} full products (median {t:.3f} s) of the same workload: {what}"}


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU product path timed on the host cores."""
    if rank != 0:
        return
    from cbm import cbm_mkl_cpp
    from oracle import oracle

    ei, n, spec = load_graph(0, 1)
    s = cbm_mkl_cpp.build_cached(ei[0], ei[1], n, spec["alpha"], CACHE)
    crow, col = s.csr_ptr, s.csr_col
    deg = np.diff(oracle.csr_from_edges(ei, n)[0]).astype(np.float32)
    with np.errstate(divide="ignore"):
        dinv = (1.0 / np.sqrt(deg)).astype(np.float32)
    rows = np.repeat(np.arange(n), np.diff(crow))
    val = (s.csr_val * dinv[col]) * dinv[rows]
    x = np.random.default_rng(1).standard_normal((n, COLS), dtype=np.float32)
    z, e, b = int(col.size), int(s.src.size), int(s.branches.size) - 1
    b_alg = bytes_alg(n, z, e, b, COLS)
    run, kind, what = reference_cpu_product()
    for _ in range(args.warmup):
        run(crow, col, val, x, s.branches, s.src, s.dst, dinv)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        run(crow, col, val, x, s.branches, s.src, s.dst, dinv)
        ts.append(time.perf_counter() - t0)
    t = sum(ts) / len(ts)
    v = b_alg / t / 1e9
    line = {"impl": "reference", "metric": "CBM DAD.X GB/s (algorithmic bytes)", "value": v, "unit": "GB/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config_dict(n, s.nnz_a, z, e, b, world),
            "cpu_baseline": {"value": v, "unit": "GB/s", "cores": host_threads(), "kind": kind,
                             "sample": f"every step one full product of the workload: {what}"},
            "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_forms:
        # context beside the CPU arm: the reference's GPU path on this box
        line["reference_gpu"] = _form(lambda: reference_gpu_timing(
            args.steps, args.warmup, (n, crow, col, val, s.branches, s.src, s.dst, dinv, x, b_alg)))
    print(json.dumps(line), flush=True)


def gcn_timing(steps, warmup):
    """2-layer GCN (128 -> 256 -> 40) on the 170,000-node power-law graph: forward +
    backward ms per step, BF16 activations vs plain FP32 (cbm4dad adjacency),
    eager and replayed from a CUDA graph of the whole step."""
    from cbm import _lib, synthetic
    from cbm.cbm4dad import cbm4dad
    from cbm.gcn import GCN, cross_entropy

    ei, n, spec = synthetic.workload("powerlaw-170k")
    a = cbm4dad(torch.from_numpy(ei), torch.ones(ei.shape[1]), alpha=spec["alpha"], cache_dir=CACHE)
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn(n, 128, device="cuda", generator=g)
    labels = torch.randint(0, 40, (n,), device="cuda", generator=g)
    out = {"workload": "powerlaw-170k GCN 128-256-40, fwd+bwd, cross-entropy on uniform labels",
           "nodes": n, "nnz_a": int(a.structure_stats["nnz_a"]), "nnz_delta": int(a.structure_stats["nnz_delta"])}
    for name, dt in (("bf16", torch.bfloat16), ("fp32", torch.float32)):
        model = GCN(a, 128, 256, 40, act_dtype=dt)
        xin = x.to(dt)

        def step():
            model.w1.grad = None
            model.w2.grad = None
            loss = cross_entropy(model(xin), labels)
            loss.backward()

        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        l0 = a.plan.stat(_lib.P_LAUNCHES)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            step()
        e1.record()
        torch.cuda.synchronize()
        out[f"{name}_ms"] = e0.elapsed_time(e1) / steps
        out[f"{name}_cbm_launches_per_step"] = (a.plan.stat(_lib.P_LAUNCHES) - l0) / steps
        # the same step captured once as a CUDA graph (forward, loss and
        # backward; the weight gradients are the graph's outputs) and replayed
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            for _ in range(3):
                step()
        torch.cuda.current_stream().wait_stream(s)
        model.w1.grad = None
        model.w2.grad = None
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            cross_entropy(model(xin), labels).backward()
        out[f"{name}_graph_ms"] = _time_events(graph.replay, steps, warmup)
        del graph
        # the step's CBM work alone: Ahat X (128 columns), Ahat (H W2) (40 columns,
        # FP32 out) and the adjoint of the latter, on the step's dtypes
        x_act = xin
        y128 = torch.empty(n, 128, dtype=dt, device="cuda")
        hw = torch.randn(n, 40, device="cuda", generator=g).to(dt)
        y40 = torch.empty(n, 40, device="cuda")
        g40 = torch.randn(n, 40, device="cuda", generator=g)
        dx40 = torch.empty(n, 40, device="cuda")  # FP32 gradient in, FP32 out (as autograd runs it)

        def backward_40():
            # what the autograd backward runs: Ahat is symmetric, so Ahat^T g = Ahat g
            if a.self_adjoint:
                a.matmul(g40, dx40)
            else:
                a.adjoint(g40, dx40)

        def cbm_work():
            a.matmul(x_act, y128)
            a.matmul(hw, y40)
            backward_40()

        out[f"{name}_cbm_ms"] = _time_events(cbm_work, steps, warmup)
        out[f"{name}_cbm_parts_ms"] = {
            "ahat_x_128": _time_events(lambda: a.matmul(x_act, y128), steps, warmup),
            "ahat_hw_40": _time_events(lambda: a.matmul(hw, y40), steps, warmup),
            "backward_40": _time_events(backward_40, steps, warmup),
            "adjoint_kernels_40": _time_events(lambda: a.adjoint(g40, dx40), steps, warmup)}
    out["speedup_bf16_over_fp32"] = out["fp32_ms"] / out["bf16_ms"]
    out["cbm_speedup_bf16_over_fp32"] = out["fp32_cbm_ms"] / out["bf16_cbm_ms"]
    out["backward_uses_forward"] = bool(a.self_adjoint)
    a.plan.check_device()
    return out


def _time_events(fn, steps, warmup):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


BATCH_SPACE = {"chunk_nnz": [128, 256], "rows_per_claim": [2, 4, 8], "variant": ["auto", "register"], "team": [0, 8]}
PREC_SPACE = {"chunk_nnz": [256, 512], "rows_per_claim": [4, 8, 16], "variant": ["auto", "register", "tma"],
              "hot_rows": [0, 65536, 262144]}


def batch_form(steps, warmup, space=None):
    """Batching form: 512 community graphs (log-uniform 1,000..64,000 nodes, mean
    degree U[8, 40], seed 4) in one launch replayed from a CUDA graph;
    D^-1/2 A D^-1/2 X with X [sum N, 64] BF16, Y FP32; launch knobs autotuned
    over ``space``."""
    from cbm import _lib, synthetic
    from cbm.batch import cbm_batch
    from cbm.tune import autotune

    t0 = time.time()
    graphs = synthetic.batch_graphs(512, seed=4)
    b = cbm_batch(graphs, alpha=0, op="dadx")
    setup_s = time.time() - t0
    n = b.num_nodes
    g = torch.Generator(device="cuda").manual_seed(4)
    x = torch.randn(n, 64, device="cuda", generator=g).to(torch.bfloat16)
    y = torch.empty(n, 64, device="cuda")
    tuned = autotune(b.plan, "dadx", x, y, space=space or BATCH_SPACE)
    l0 = b.plan.stat(_lib.P_LAUNCHES)
    b.matmul(x, y)  # kernels one product launches (the replay launches the same)
    launches = b.plan.stat(_lib.P_LAUNCHES) - l0
    graph = b.capture(x, y)
    ms = _time_events(graph.replay, steps, warmup)
    st = b.plan.stats
    b_alg = bytes_alg(n, st["nnz"], st["edges"], st["branches"], 64, sx=2, sy=4)
    b_min = bytes_compulsory(n, st["nnz"], st["edges"], st["branches"], 64, sx=2, sy=4)
    offs = b.offsets
    packed = np.concatenate([np.asarray(ei, dtype=np.int64) + int(offs[i]) for i, (ei, _) in enumerate(graphs)],
                            axis=1)
    dinv = dinv_f64(packed, n)
    err = fp64_sample_error(packed, n, x, y, rs=dinv, cs=dinv)
    b.plan.check_device()
    del graph
    return {"metric": "CBM batched DAD.X GB/s (algorithmic bytes)", "value": b_alg / (ms * 1e-3) / 1e9,
            "unit": "GB/s", "ms": ms, "steps": steps, "warmup": warmup,
            "dtype": "bf16 X, f32 Y, f32 accumulate",
            "config": {"workload": "512 community graphs, one launch under a CUDA graph", "graphs": len(graphs),
                       "nodes": n, "nnz_a": b.nnz_a, "nnz_delta": st["nnz"], "tree_edges": st["edges"],
                       "cols": 64, "setup_s": setup_s},
            "graphs_per_s": len(graphs) / (ms * 1e-3), "rows_per_s": n / (ms * 1e-3),
            "kernels_per_replay": launches, "autotune_best": {"config": tuned[0][0], "ms": tuned[0][1]},
            "roofline": roofline(b_alg, b_min, ms), "error_vs_fp64": err}


def run_batch(args):
    r = batch_form(args.steps, args.warmup)
    line = {"metric": r.pop("metric"), "value": r.pop("value"), "unit": r.pop("unit"), "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r.pop("ms"), "higher_is_better": True,
            "data": "synthetic"}
    line.update(r)
    print(json.dumps(line), flush=True)


def precision_form(steps, warmup, prec_nodes=0, space=None, knobs=None):
    """Precision form: A D^-1/2 X on the 2,400,000-node power-law graph
    (exponent 2.3, mean degree 50, 40% near-duplicate rows with 5% flips, seed 2,
    alpha 16); X [N, 128] stored BF16, FP32 accumulation and output.  Launch
    knobs from ``knobs`` or autotuned over ``space``."""
    from cbm import synthetic
    from cbm.cbm4ad import cbm4ad

    t0 = time.time()
    if prec_nodes:
        # the same law at another size (profiling runs)
        n = prec_nodes
        ei = synthetic._w_powerlaw(n, 2.3, 50.0, 0.40, 0.05, 2)
        spec = {"alpha": 16}
    else:
        ei, n, spec = synthetic.workload("powerlaw-2.4m")
    a = cbm4ad(torch.from_numpy(ei), torch.ones(ei.shape[1]), alpha=spec["alpha"], cache_dir=CACHE)
    setup_s = time.time() - t0
    g = torch.Generator(device="cuda").manual_seed(2)
    x32 = torch.randn(n, 128, device="cuda", generator=g)
    x = x32.to(torch.bfloat16)
    y = torch.empty(n, 128, device="cuda")
    tuned = None
    if knobs is not None:
        a.plan.tune(**knobs)
    else:
        from cbm.tune import autotune

        tuned = autotune(a.plan, "adx", x, y, space=space or PREC_SPACE)
    ms = _time_events(lambda: a.matmul(x, y), steps, warmup)
    dinv = dinv_f64(ei, n)
    err = {"product": fp64_sample_error(ei, n, x, y, cs=dinv),
           "end_to_end": fp64_sample_error(ei, n, x32, y, cs=dinv)}
    st = a.plan.stats
    b_alg = bytes_alg(n, st["nnz"], st["edges"], st["branches"], 128, sx=2, sy=4)
    b_min = bytes_compulsory(n, st["nnz"], st["edges"], st["branches"], 128, sx=2, sy=4)
    a.plan.check_device()
    return {"metric": "CBM A.D^-1/2.X GB/s (algorithmic bytes), BF16 X", "value": b_alg / (ms * 1e-3) / 1e9,
            "unit": "GB/s", "ms": ms, "steps": steps, "warmup": warmup,
            "dtype": "bf16 X, f32 Y, f32 accumulate",
            "config": {"workload": f"powerlaw (exponent 2.3, mean degree 50, 40% near-duplicates) N={n} A D^-1/2 X",
                       "nodes": n, "nnz_a": a.structure_stats["nnz_a"], "nnz_delta": st["nnz"],
                       "tree_edges": st["edges"], "cols": 128, "alpha": spec["alpha"], "setup_s": setup_s},
            "rows_per_s": n / (ms * 1e-3), "roofline": roofline(b_alg, b_min, ms), "plan": st,
            "autotune_best": {"config": tuned[0][0], "ms": tuned[0][1]} if tuned else {"config": knobs},
            "error_vs_fp64": err}


def run_precision(args):
    knobs = None
    if args.no_autotune:
        knobs = dict(chunk_nnz=args.chunk_nnz, rows_per_claim=args.rows_per_claim, variant=args.variant,
                     hot_rows=args.hot_rows, team=args.team)
    r = precision_form(args.steps, args.warmup, prec_nodes=args.prec_nodes, knobs=knobs)
    line = {"metric": r.pop("metric"), "value": r.pop("value"), "unit": r.pop("unit"), "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r.pop("ms"), "higher_is_better": True,
            "data": "synthetic"}
    line.update(r)
    print(json.dumps(line), flush=True)


def direct_form(a, x, y_plan, b_alg, plan_ms, steps, warmup, ei, n):
    """The reference's CPU operator s_spmm_fused_update_csr_int32
    (cbm/cbm_extensions.cpp:593-698) through its own signature on CUDA tensors
    (csrc/direct.cu: no plan; the caller's CSR and tree arrays read as given),
    on the headline's structure, prepared values, multipliers and X: ms per
    product at the headline's algorithmic bytes, beside the plan path; its
    error against FP64 on sampled rows, and its largest difference from the
    plan path's result.  The two sum a row's entries in different orders
    (one sequential chain here, chunk partials added in order for the plan's
    long rows) and round the update differently (fma(Y[u], m[v] / m[u], Y[v])
    here, as the CPU code does), so they agree to rounding, not bit for bit."""
    from cbm import cbm_mkl_cpp

    crow = a.deltas.crow_indices()
    rp_b, rp_e = crow[:-1], crow[1:]
    col, val = a.deltas.col_indices(), a.deltas.values()
    out = torch.empty_like(y_plan)

    def run():
        cbm_mkl_cpp.s_spmm_fused_update_csr_int32(rp_b, rp_e, col, val, x, a.mca_offset, a.mca_src_idx,
                                                  a.mca_dst_idx, a.D, out)

    ms = _time_events(run, steps, warmup)
    run()
    torch.cuda.synchronize()
    cbm_mkl_cpp.check_device()
    max_diff = float((out - y_plan).abs().max())
    dinv = dinv_f64(ei, n)
    err = fp64_sample_error(ei, n, x, out, rs=dinv, cs=dinv)
    del out
    return {"call": "cbm_mkl_cpp.s_spmm_fused_update_csr_int32 on CUDA tensors (the reference's operator "
                    "signature, stateless GPU product)",
            "ms": ms, "value": b_alg / (ms * 1e-3) / 1e9, "unit": "GB/s", "plan_ms": plan_ms,
            "error_vs_fp64": err, "max_abs_diff_vs_plan": max_diff}


def small_form(steps, warmup):
    """The 4,096-node community graph (64 communities of 64, 12 in-community
    and 4 uniform neighbours, seed 0, alpha 0): A.X with X FP32 U[-1, 1],
    4096 x 64.  The operands (1 MB) sit in L2, so this times launch latency,
    not memory: one eager call and one CUDA-graph replay of the same call.
    The reference's GPU path on the same graph is timed by --impl reference."""
    from cbm import synthetic
    from cbm.cbm4mm import cbm4mm

    ei, n, spec = synthetic.workload("community-4096")
    a = cbm4mm(torch.from_numpy(ei), torch.ones(ei.shape[1]), alpha=0)
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.rand(n, 64, device="cuda", generator=g) * 2 - 1
    y = torch.empty_like(x)
    st = a.plan.stats
    b_alg = bytes_alg(n, st["nnz"], st["edges"], st["branches"], 64, scaled=False)
    reps = 20  # products per timed replay or loop, so each event pair spans many launches
    eager_ms = _time_events(lambda: [a.matmul(x, y) for _ in range(reps)], steps, warmup) / reps
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(3):
            a.matmul(x, y)
    torch.cuda.current_stream().wait_stream(s)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        for _ in range(reps):
            a.matmul(x, y)
    graph_ms = _time_events(graph.replay, steps, warmup) / reps
    out = {"workload": "community-4096 A.X (c0 shape: 4096 nodes, 64 FP32 columns, alpha 0)", "nodes": n,
           "nnz_a": int(a.structure_stats["nnz_a"]), "nnz_delta": int(st["nnz"]),
           "eager_us": eager_ms * 1e3, "graph_replay_us": graph_ms * 1e3,
           "graph_replay_gbs": b_alg / (graph_ms * 1e-3) / 1e9,
           "note": "L2-resident and launch-bound: no roofline claim"}
    a.plan.check_device()
    return out


def reference_gpu_timing(steps, warmup, headline):
    """The reference's own GPU products (cbm/cbm.cu, compiled from its source
    into oracle/_ref/ by oracle/build_ref.py), timed with CUDA events on the
    structures this arm's CPU leg uses: matmul_DAX_DADX (cuSPARSE SpMM, then
    its fused_update kernel) on the headline workload, and matmul_AX_ADX on the
    4,096-node community graph (A.X, 64 FP32 columns, eager: its per-call
    allocations keep it out of CUDA graphs).  ``headline`` = (n, crow, col,
    val, branches, src, dst, dinv, x, b_alg) as host arrays."""
    from oracle import build_ref

    if not torch.cuda.is_available():
        return {"unavailable": "no GPU"}
    mod = build_ref.load("cbm_cusparse_ref")
    if mod is None:
        return {"unavailable": "the reference's GPU module was not built (no reference tree at build time)"}
    dev = torch.device("cuda")

    def make(n, crow, col, val, br, src, dst, mult):
        t = lambda a, d: torch.from_numpy(np.ascontiguousarray(a, dtype=d)).to(dev)
        csr = torch.sparse_csr_tensor(t(crow, np.int32), t(col, np.int32), t(val, np.float32), (n, n))
        # its update kernel reads one branch offset past the end (one block per
        # entry of mca_branches, cbm/cbm.cu:136, :193): a view of a buffer with
        # a readable sentinel equal to the edge count
        brp = t(np.append(br, br[-1]), np.int32)[: len(br)]
        m = t(mult, np.float32) if mult is not None else torch.empty(0, device=dev)
        s_t, d_t = t(src, np.int32), t(dst, np.int32)
        # the extension keeps raw pointers to every tensor it is given
        # (cbm/cbm.cu:110-140): all of them must outlive it
        return mod.cusparseCBM(csr, brp, s_t, d_t, m), (csr, brp, m, s_t, d_t)

    out = {"impl": "reference cusparseCBM (cbm/cbm.cu), built from its source for sm_100a"}
    n, crow, col, val, br, src, dst, dinv, x, b_alg = headline
    ref, keep = make(n, crow, col, val, br, src, dst, dinv)
    xt = torch.from_numpy(x).to(dev)
    y = torch.empty_like(xt)
    ms = _time_events(lambda: ref.matmul_DAX_DADX(xt, y), max(steps, 10), max(warmup, 3))
    out["headline"] = {"call": "matmul_DAX_DADX", "ms": ms, "value": b_alg / (ms * 1e-3) / 1e9, "unit": "GB/s"}
    del ref, keep, xt, y
    from cbm import cbm_mkl_cpp, synthetic

    ei, n, _ = synthetic.workload("community-4096")
    st = cbm_mkl_cpp.build(ei[0], ei[1], n, 0)
    ref, keep = make(n, st.csr_ptr, st.csr_col, st.csr_val, st.branches, st.src, st.dst, None)
    g = torch.Generator(device="cuda").manual_seed(0)
    xs = torch.rand(n, 64, device=dev, generator=g) * 2 - 1
    ys = torch.empty_like(xs)
    reps = 20
    ms = _time_events(lambda: [ref.matmul_AX_ADX(xs, ys) for _ in range(reps)], max(steps, 10),
                      max(warmup, 3)) / reps
    out["small"] = {"call": "matmul_AX_ADX", "workload": "community-4096 A.X, 64 FP32 columns", "us": ms * 1e3}
    del ref, keep
    return out


def run_lsh(args):
    """LSH-clustered form: the rows of the 1,000,000-node power-law graph are
    clustered by the reference's hierarchical fingerprinting
    (benchmark/clustering_gpu.py, 4 hash columns, clusters of at most
    args.max_cluster rows), one CBM forest per cluster in one structure, and
    D^-1/2 A D^-1/2 X (fp32, 256 columns) runs over all clusters in one launch.
    Reports the reference's compression figures next to the timing."""
    from cbm import synthetic
    from cbm.cbm4dad import cbm4dad
    from cbm.cluster import cluster_ids, lsh_clusters

    ei, n, spec = load_graph(0, 1)
    t0 = time.time()
    cl = lsh_clusters(ei, n, max_cluster_size=args.max_cluster, num_hashes=4)
    t_cluster = time.time() - t0
    a = cbm4dad(torch.from_numpy(ei), torch.ones(ei.shape[1]), alpha=spec["alpha"], cache_dir=CACHE,
                cluster=cluster_ids(cl, n))
    full = cbm4dad(torch.from_numpy(ei), torch.ones(ei.shape[1]), alpha=spec["alpha"], cache_dir=CACHE)
    g = torch.Generator(device="cuda").manual_seed(1)
    x = torch.randn(n, COLS, device="cuda", generator=g)
    y = torch.empty(n, COLS, device="cuda")
    ms = _time_events(lambda: a.matmul(x, y), args.steps, args.warmup)
    ms_full = _time_events(lambda: full.matmul(x, y), args.steps, args.warmup)
    a.matmul(x, y)
    st = a.plan.stats
    b_alg = bytes_alg(n, st["nnz"], st["edges"], st["branches"], COLS)
    d = dinv_f64(ei, n)
    sizes = sorted(c.size for c in cl)
    line = {"metric": "CBM DAD.X GB/s over LSH clusters (algorithmic bytes)", "value": b_alg / (ms * 1e-3) / 1e9,
            "unit": "GB/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{WORKLOAD} rows in LSH clusters (4 hashes, <= {args.max_cluster} rows), "
                                   f"one launch", "nodes": n, "cols": COLS, "clusters": len(cl),
                       "cluster_rows_min_median_max": [sizes[0], sizes[len(sizes) // 2], sizes[-1]],
                       "clustering_s": t_cluster},
            "compression": {"nnz_csr": a.structure_stats["nnz_a"], "nnz_cbm": full.structure_stats["nnz_delta"],
                            "nnz_cbm_clustered": st["nnz"],
                            "reduction_vs_csr": a.structure_stats["nnz_a"] / st["nnz"],
                            "reduction_vs_cbm": full.structure_stats["nnz_delta"] / st["nnz"]},
            "unclustered_ms": ms_full,
            "roofline": {"bound": "hbm", "achieved": b_alg / (ms * 1e-3) / 1e9, "peak": peaks()[0], "unit": "GB/s",
                         "frac": b_alg / (ms * 1e-3) / 1e9 / peaks()[0], "peak_kind": peaks()[1]},
            "error_vs_fp64": fp64_sample_error(ei, n, x, y, rs=d, cs=d)}
    a.plan.check_device()
    print(json.dumps(line), flush=True)


def _form(fn):
    """One of the other forms' records; a failure is recorded, not raised, so
    that the headline line still prints."""
    try:
        return fn()
    except Exception as exc:  # recorded in the line for the reader
        return {"error": f"{type(exc).__name__}: {exc}"}


def config_dict(n, nnz_a, z, e, b, world):
    return {"workload": f"{WORKLOAD}: D^-1/2 A D^-1/2 X fp32, power-law N={n}, alpha=8, C={COLS} per GPU",
            "nodes": n, "nnz_a": nnz_a, "nnz_delta": z, "tree_edges": e, "branches": b, "cols_per_gpu": COLS,
            "l2": "inputs larger than L2 (X and Y 1.02 GB each), no flush", "parallelism": f"column shards x{world}"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-gcn", action="store_true")
    ap.add_argument("--no-forms", action="store_true",
                    help="leave the precision, batch and reference-GPU records out of the headline line")
    ap.add_argument("--gcn-only", action="store_true", help="only the GCN timing (one JSON object)")
    ap.add_argument("--workload", default="headline", choices=["headline", "batch", "precision", "lsh", "small"],
                    help="batch / precision / lsh: the batching, precision or LSH-clustered form instead of "
                         "the headline line")
    ap.add_argument("--max-cluster", type=int, default=100000, help="lsh workload: cluster size bound")
    ap.add_argument("--variant", default="auto", choices=["auto", "register", "staged"])
    ap.add_argument("--chunk-nnz", type=int, default=256)
    ap.add_argument("--rows-per-claim", type=int, default=4)
    ap.add_argument("--team", type=int, default=0)
    ap.add_argument("--hot-rows", type=int, default=65536)
    ap.add_argument("--slab-cols", type=int, default=64, help="column slab of the host-operand product (e2e)")
    ap.add_argument("--prec-nodes", type=int, default=0, help="precision workload at this many nodes (same law)")
    ap.add_argument("--no-autotune", action="store_true", help="precision workload: the given knobs, no autotuning")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                             device_id=torch.device("cuda", local))
    if args.impl == "reference":
        run_reference(args, rank, world)
        if world > 1:
            torch.distributed.destroy_process_group()
        return

    from cbm import _lib
    from cbm.cbm4dad import cbm4dad

    if args.workload != "headline":
        if rank == 0:
            {"batch": run_batch, "precision": run_precision, "lsh": run_lsh,
             "small": lambda a: print(json.dumps(small_form(a.steps, max(a.warmup, 3))), flush=True)}[
                args.workload](args)
        return
    if args.gcn_only:
        if rank == 0:
            print(json.dumps(gcn_timing(max(args.steps, 10), max(args.warmup, 3))), flush=True)
        return

    from cbm.shard import column_shard, max_over_ranks

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    ei, n, spec = load_graph(rank, world)
    # weak scaling: rank r owns columns [c0, c1) of a [N, COLS * world] X and Y
    c0, c1 = column_shard(COLS * world, rank, world)
    assert c1 - c0 == COLS
    # rank 0 constructs the CBM into the cache first; the others then load it
    # (every rank takes the one barrier)
    if world > 1 and rank != 0:
        torch.distributed.barrier()
    a = cbm4dad(torch.from_numpy(ei), torch.ones(ei.shape[1]), alpha=spec["alpha"], cache_dir=CACHE)
    if world > 1 and rank == 0:
        torch.distributed.barrier()
    a.plan.tune(chunk_nnz=args.chunk_nnz, rows_per_claim=args.rows_per_claim, variant=args.variant,
                hot_rows=args.hot_rows, team=args.team)
    st = a.plan.stats
    z, e, b = st["nnz"], st["edges"], st["branches"]
    b_alg = bytes_alg(n, z, e, b, COLS)

    g = torch.Generator(device=dev).manual_seed(1 + rank)
    x = torch.randn(n, COLS, device=dev, generator=g)
    y = torch.empty(n, COLS, device=dev)
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(dev)

    # ---- device-timed product (inputs resident in HBM) ----
    for _ in range(args.warmup):
        a.matmul(x, y)
    barrier()
    launches0 = a.plan.stat(_lib.P_LAUNCHES)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with Clocks(local) as clk:
        barrier()
        evs[0].record(stream)
        for i in range(args.steps):
            a.matmul(x, y)
            evs[i + 1].record(stream)
        barrier()
    launches = a.plan.stat(_lib.P_LAUNCHES) - launches0
    per = [evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps)]
    ms = evs[0].elapsed_time(evs[-1]) / args.steps
    ms_max = max_over_ranks(ms, dev)
    a.plan.check_device()
    err = fp64_sample_error(ei, n, x, y, rs=dinv_f64(ei, n), cs=dinv_f64(ei, n)) if rank == 0 else None

    # ---- end to end through the public API with host buffers ----
    # cbm4dad.matmul_host: X copied in and Y copied out in column slabs, the
    # copies of one slab overlapped with the product of another
    xh = torch.empty(n, COLS, dtype=torch.float32, pin_memory=True)
    xh.copy_(x.cpu())
    yh = torch.empty(n, COLS, dtype=torch.float32, pin_memory=True)
    # back-to-back steps overlap one step's copy-out with the next step's
    # copy-in (overlap_calls); every step still copies its X in and its Y
    # out inside the timed region, which ends after the last copy-out
    # (host_wait)
    e2e_steps = max(3, min(args.steps, 10))
    for _ in range(2):
        a.matmul_host(xh, yh, slab_cols=args.slab_cols, overlap_calls=True)
    a.host_wait()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        a.matmul_host(xh, yh, slab_cols=args.slab_cols, overlap_calls=True)
    a.host_wait()
    e1.record(stream)
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / e2e_steps, dev)
    # the PCIe bound of one step: the same bytes copied in and out at once
    # (pinned host <-> HBM, one stream each way) with no product; x and y
    # get back the values they hold
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    copy_ms = []
    for i in range(5):
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        s_in.wait_stream(stream)
        s_out.wait_stream(stream)
        with torch.cuda.stream(s_in):
            x.copy_(xh, non_blocking=True)
        with torch.cuda.stream(s_out):
            yh.copy_(y, non_blocking=True)
        stream.wait_stream(s_in)
        stream.wait_stream(s_out)
        c1.record(stream)
        c1.synchronize()
        if i >= 2:
            copy_ms.append(c0.elapsed_time(c1))
    copy_ms = max_over_ranks(statistics.mean(copy_ms), dev)

    if rank == 0:
        kernel_ms = statistics.mean(per)
        traffic, traffic_src = traffic_from_profile()
        rl = roofline(b_alg, bytes_compulsory(n, z, e, b, COLS), kernel_ms, traffic)
        rl["kernel"] = ("cbm::fwd_kernel<float,float,2,4>" if args.variant == "register"
                        else "cbm::fwd_stream_kernel<float,float,32,2,4,8,128>")
        rl["traffic_source"] = traffic_src
        line = {
            "metric": "CBM DAD.X GB/s (algorithmic bytes)",
            "value": b_alg * world / (ms_max * 1e-3) / 1e9,
            "unit": "GB/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_max,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": config_dict(n, a.structure_stats["nnz_a"], z, e, b, world),
            "rows_per_s": n * world / (ms_max * 1e-3),
            "roofline": rl,
            "e2e": {"value": b_alg * world / (e2e_ms * 1e-3) / 1e9, "unit": "GB/s",
                    "h2d_bytes_per_step": int(xh.numel() * 4), "d2h_bytes_per_step": int(yh.numel() * 4),
                    "ms_per_step": e2e_ms,
                    "copy_bound_ms": copy_ms,
                    "frac_of_copy_bound": copy_ms / e2e_ms,
                    "api": "cbm4dad.matmul_host (pinned host X and Y, overlap_calls=True)",
                    "slab_cols": args.slab_cols},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "plan": a.plan.stats,
            "error_vs_fp64": err,
        }
        if not args.no_gcn:
            line["gcn"] = gcn_timing(max(args.steps, 10), max(args.warmup, 3))
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(a, x.cpu().numpy(), b_alg)
        if world == 1 and not args.no_forms:
            # y holds the plan product of x (the last step of the e2e leg wrote
            # y_host, not y)
            line["direct"] = _form(lambda: direct_form(a, x, y, b_alg, kernel_ms, max(args.steps, 10), args.warmup,
                                                       ei, n))
        if world == 1 and not args.no_forms:
            del xh, yh, x, y, a
            torch.cuda.empty_cache()
            line["precision"] = _form(lambda: precision_form(max(args.steps, 10), args.warmup,
                                                             space={"chunk_nnz": [256, 512],
                                                                    "rows_per_claim": [8, 16],
                                                                    "hot_rows": [0, 65536]}))
            torch.cuda.empty_cache()
            line["batch"] = _form(lambda: batch_form(max(args.steps, 10), args.warmup))
            line["small"] = _form(lambda: small_form(max(args.steps, 10), max(args.warmup, 3)))
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
