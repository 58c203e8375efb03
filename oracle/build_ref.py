"""Compiles the reference's own GPU product path into oracle/_ref/ -- TEST INFRASTRUCTURE ONLY.

Sources are read where they lie, /root/reference/cbm/cbm.cu (module
cbm_cusparse: cusparseCBM, cbm/cbm.cu:93-310) and /root/reference/cbm/csr.cu
(module csr_cusparse: cusparseCSR, cbm/csr.cu:24-133).  Both need only torch's
extension headers and cuSPARSE from the CUDA toolkit; they are compiled for
sm_100a with torch.utils.cpp_extension into oracle/_ref/ (git-ignored; the built
.so files travel with the repository snapshot to the GPU machine, where the
GPU tests load them as a second checker).  Nothing is copied from the
reference tree.

The reference's own setup scripts are not run (cbm/setup_cbm_cusparse.py).
cbm/cbm_extensions.cpp (the CPU constructor and CPU products) is not built: it
needs Intel MKL headers/libraries and the arbok submodule, neither present.
"""
from __future__ import annotations

import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SRC = "/root/reference/cbm"
OUT = os.path.join(HERE, "_ref")
MODULES = {"cbm_cusparse_ref": "cbm.cu", "csr_cusparse_ref": "csr.cu"}


def build(verbose=False):
    if not os.path.isdir(REF_SRC):
        return []
    os.makedirs(OUT, exist_ok=True)
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0a")
    from torch.utils import cpp_extension

    built = []
    for name, src in MODULES.items():
        so = os.path.join(OUT, name + ".so")
        srcp = os.path.join(REF_SRC, src)
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
    return built


def load(name):
    """Imports a built reference module (torch must be importable); None if absent."""
    import importlib.util

    import torch  # noqa: F401  (the module's symbols live in torch's libraries)

    so = os.path.join(OUT, name + ".so")
    if not os.path.exists(so):
        return None
    spec = importlib.util.spec_from_file_location(name, so)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
