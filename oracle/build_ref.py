"""Compiles the reference's own product code into oracle/_ref/ -- TEST INFRASTRUCTURE ONLY.

Sources are read where they lie in the reference tree (cbm4scale/CBM-GPU),
whose root comes from the ``ref_dir`` argument, else the CBM_REFERENCE_DIR
environment variable, else the tree mounted read-only on the build machine.
Nothing is copied from it; the built files are git-ignored and travel with
the repository snapshot to the GPU machine, where tests and the bench's
baseline legs load them as checkers and baselines, never as the product.

GPU path (torch.utils.cpp_extension, sm_100a):
  cbm_cusparse_ref.so   cbm/cbm.cu (cusparseCBM, cbm/cbm.cu:93-310)
  csr_cusparse_ref.so   cbm/csr.cu (cusparseCSR, cbm/csr.cu:24-133)
Both need only torch's extension headers and cuSPARSE.

CPU path (g++ directly, this recipe):
  cbm_mkl_cpp_ref.so    cbm/cbm_extensions.cpp: the reference's eight MKL
                        product operators (:351-907, bound at :909-919)
cbm_extensions.cpp includes mkl.h, mkl_spblas.h and arbok's tarjan_pq.h,
none of which is present.  oracle/ref_shim/ holds project-written
declarations of the names it uses (MKL's published LP64 C API; one arbok
class), no definitions.  The products need mkl_sparse_s_create_csr,
mkl_sparse_s_mm, mkl_sparse_destroy and cblas_saxpy, which libtorch_cpu.so
exports; the module links against it.  The constructor cbm_init_ also needs
mkl_sparse_syrk, mkl_sparse_s_create_coo, mkl_sparse_convert_csr and arbok,
which nothing here provides, so the module is linked with lazy binding,
loaded with RTLD_LAZY and its ``init`` is never called.  Before the module is
trusted, ref_shim/mkl_kat.c (a known-answer 3x3 SpMM, its transpose and a
saxpy through the same declarations) must pass in a child process.

The reference's own setup scripts are not run.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SHIM = os.path.join(HERE, "ref_shim")
MODULES = {"cbm_cusparse_ref": "cbm.cu", "csr_cusparse_ref": "csr.cu"}
CPU_MODULE = "cbm_mkl_cpp_ref"


def reference_dir(ref_dir=None):
    """Root of the reference tree (the directory holding cbm/)."""
    return ref_dir or os.environ.get("CBM_REFERENCE_DIR") or "/root/reference"


def _torch_paths():
    import sysconfig

    import torch
    from torch.utils import cpp_extension

    return (cpp_extension.include_paths(), cpp_extension.library_paths()[0], sysconfig.get_paths()["include"],
            int(torch._C._GLIBCXX_USE_CXX11_ABI))


def mkl_kat(verbose=False):
    """Builds and runs the known-answer check of libtorch_cpu's MKL entry points
    in a child process; True if it passes."""
    _, torch_lib, _, _ = _torch_paths()
    os.makedirs(OUT, exist_ok=True)
    exe = os.path.join(OUT, "mkl_kat")
    cmd = ["gcc", "-O1", "-I" + SHIM, os.path.join(SHIM, "mkl_kat.c"), "-o", exe, "-L" + torch_lib, "-ltorch_cpu",
           "-Wl,-rpath," + torch_lib]
    if subprocess.run(cmd, capture_output=not verbose).returncode != 0:
        return False
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    if verbose:
        print(r.stdout, r.stderr)
    return r.returncode == 0


def build_cpu(ref_dir=None, verbose=False):
    """The reference's MKL CPU operators as oracle/_ref/cbm_mkl_cpp_ref.so; None
    if the reference tree is absent or the known-answer check fails."""
    src = os.path.join(reference_dir(ref_dir), "cbm", "cbm_extensions.cpp")
    if not os.path.exists(src):
        return None
    so = os.path.join(OUT, CPU_MODULE + ".so")
    deps = [src] + [os.path.join(SHIM, f) for f in ("mkl.h", "mkl_spblas.h", "mkl_kat.c")]
    if os.path.exists(so) and all(os.path.getmtime(so) >= os.path.getmtime(d) for d in deps):
        return so
    if not mkl_kat(verbose):
        return None
    includes, torch_lib, py_include, abi = _torch_paths()
    os.makedirs(OUT, exist_ok=True)
    tmp = so + ".tmp"
    cmd = (["g++", "-O2", "-std=c++20", "-fopenmp", "-mavx2", "-mfma", "-fPIC", "-shared", "-w",
            f"-D_GLIBCXX_USE_CXX11_ABI={abi}", f"-DTORCH_EXTENSION_NAME={CPU_MODULE}",
            "-DTORCH_API_INCLUDE_EXTENSION_H", "-I" + SHIM] + ["-I" + p for p in includes] +
           ["-I" + py_include, src, "-o", tmp, "-L" + torch_lib, "-ltorch_cpu", "-ltorch", "-lc10", "-ltorch_python",
            "-Wl,-z,lazy", "-Wl,-rpath," + torch_lib])
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        if verbose:
            print(r.stdout, r.stderr)
        return None
    os.replace(tmp, so)
    return so


def build(verbose=False, ref_dir=None):
    root = reference_dir(ref_dir)
    ref_src = os.path.join(root, "cbm")
    if not os.path.isdir(ref_src):
        return []
    os.makedirs(OUT, exist_ok=True)
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0a")
    from torch.utils import cpp_extension

    built = []
    for name, src in MODULES.items():
        so = os.path.join(OUT, name + ".so")
        srcp = os.path.join(ref_src, src)
        if os.path.exists(so) and os.path.getmtime(so) >= os.path.getmtime(srcp):
            built.append(so)
            continue
        bdir = os.path.join(OUT, "build_" + name)
        os.makedirs(bdir, exist_ok=True)
        cpp_extension.load(name=name, sources=[srcp], build_directory=bdir,
                           extra_cflags=["-O2"],
                           extra_cuda_cflags=["-O2", "-gencode", "arch=compute_100a,code=sm_100a"],
                           extra_ldflags=["-lcusparse"], verbose=verbose, is_python_module=True)
        os.replace(os.path.join(bdir, name + ".so"), so)
        built.append(so)
    cpu = build_cpu(root, verbose)
    if cpu:
        built.append(cpu)
    return built


def load(name):
    """Imports a built reference module (torch must be importable); None if absent.
    The CPU module is loaded with lazy binding (its unresolved constructor
    symbols are never bound)."""
    import importlib.util

    import torch  # noqa: F401  (the module's symbols live in torch's libraries)

    so = os.path.join(OUT, name + ".so")
    if not os.path.exists(so):
        return None
    spec = importlib.util.spec_from_file_location(name, so)
    flags = sys.getdlopenflags()
    if name == CPU_MODULE:
        sys.setdlopenflags(os.RTLD_LAZY | os.RTLD_LOCAL)
    try:
        mod = importlib.util.module_from_spec(spec)  # dlopen happens here
        spec.loader.exec_module(mod)
    finally:
        sys.setdlopenflags(flags)
    return mod


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("-")]
    print(build(verbose="-v" in sys.argv, ref_dir=args[0] if args else None))
