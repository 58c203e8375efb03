"""Builds libcbm_b200.so in-tree with nvcc for sm_100a (no torch involved).

    python -m cbm._build            (from cbm-gpu_b200/)

Sources: cbm-gpu_b200/csrc/*.cpp, *.cu (kernel instantiations split over the launch_*.cu units so
they compile in parallel); header include/.
Objects go to cbm-gpu_b200/_build/, the library next to this file.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)                 # cbm-gpu_b200/
REPO = os.path.dirname(PKG_ROOT)
CSRC = os.path.join(PKG_ROOT, "csrc")
INCLUDE = os.path.join(REPO, "include")
BUILD = os.path.join(PKG_ROOT, "_build")
LIB = os.path.join(HERE, "libcbm_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["construct.cpp", "plan.cu", "matmul.cu", "noalloc.cu", "transpose.cu", "launch_staged_f32.cu",
           "launch_staged_bf16_f32.cu", "launch_staged_bf16_bf16.cu", "launch_tma.cu", "launch_reg_f32.cu",
           "launch_reg_bf16.cu", "launch_rev.cu", "launch_tr.cu", "direct.cu"]
HEADERS = ["kernels.cuh", "plan.h", "launch.cuh"]


def _nvcc():
    cand = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    p = os.path.join(cand, "bin", "nvcc")
    return p if os.path.exists(p) else (shutil.which("nvcc") or "nvcc")


def _flags(src):
    common = ["-O3", "-std=c++17", "-I" + INCLUDE, "-I" + CSRC]
    if src.endswith(".cpp"):
        return ["-x", "c++", "-Xcompiler", "-fPIC,-fopenmp,-O3"] + common
    return ARCH + ["-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"] + common


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "cbm_b200.h")]
    jobs = []
    objs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        if force or _newer(obj, [src] + hdrs):
            jobs.append([nvcc] + _flags(s) + ["-c", src, "-o", obj])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        return r

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 8))) as ex:
        list(ex.map(run, jobs))
    if jobs or force or _newer(LIB, objs):
        run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xcompiler", "-fopenmp", "-lgomp"])
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
