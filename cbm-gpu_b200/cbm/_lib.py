"""ctypes binding of libcbm_b200.so (the C ABI in include/cbm_b200.h).

The library is loaded from this directory; there is no fallback: if it is
missing, every product raises.  Build it with ``python -m cbm._build`` (or the
repository's ``__graft_entry__.build()``).
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcbm_b200.so")

# status codes (include/cbm_b200.h)
OK, ERR_INVALID, ERR_INDEX, ERR_ALLOC, ERR_CUDA, ERR_STRUCTURE, ERR_DTYPE, ERR_SHAPE, ERR_TIMEOUT, \
    ERR_UNSUPPORTED, ERR_WORKSPACE, ERR_INTERNAL, ERR_TOO_LARGE = range(13)
NOALLOC_MAX_ROWS = 1048544
F32, BF16 = 0, 1
OP_AX, OP_ADX, OP_DADX, OP_VALUES_ADD, OP_VALUES_RATIO, OP_DAD_ADD, OP_GIN = range(7)
INPUT_DEVICE, INPUT_HOST = 0, 1
VARIANT_AUTO, VARIANT_REGISTER, VARIANT_STAGED, VARIANT_TMA = 0, 1, 2, 3
PASSES_AUTO, PASSES_FUSED, PASSES_TWO = 0, 1, 2
BUILD_EXHAUSTIVE = 1
COALESCE_SYMMETRIZE, COALESCE_DROP_SELF = 1, 2
S_DELTA_ROW, S_DELTA_COL, S_DELTA_VAL, S_BRANCHES, S_SRC, S_DST, S_PARENT, S_CSR_PTR, S_CSR_COL, \
    S_CSR_VAL = range(10)
S_N_CANDIDATES, S_TREE_COST, S_NNZ_A, S_SYMMETRIC = 100, 101, 102, 103
P_ROWS, P_COLS, P_NNZ, P_EDGES, P_BRANCHES, P_LEVELS, P_INTERNAL, P_CHUNKS, P_LONG_ROWS, P_UNIT_VALUES, \
    P_GRID, P_LAUNCHES = range(12)

vp = C.c_void_p
i32 = C.c_int32
i64 = C.c_int64

# (name, restype, argtypes): every exported symbol of include/cbm_b200.h
SIGNATURES = [
    ("cbm_build", C.c_int, [vp, vp, i64, i64, i64, i32, i32, C.POINTER(vp)]),
    ("cbm_build_clustered", C.c_int, [vp, vp, i64, i64, i64, vp, i32, i32, C.POINTER(vp)]),
    ("cbm_coalesce", C.c_int, [vp, vp, i64, i64, i32, vp, vp, C.POINTER(i64)]),
    ("cbm_structure_len", i64, [vp, i32]),
    ("cbm_structure_copy", C.c_int, [vp, i32, vp]),
    ("cbm_structure_free", None, [vp]),
    ("cbm_validate", C.c_int, [vp, vp, i64, i64, i64, vp, i64, vp, vp, i64]),
    ("cbm_plan_create", C.c_int, [vp, vp, vp, i64, i64, i64, vp, i64, vp, vp, i64, vp, i32, vp,
                                  C.POINTER(vp)]),
    ("cbm_plan_set_multipliers", C.c_int, [vp, vp, vp]),
    ("cbm_plan_tune", C.c_int, [vp, i32, i32, i32, i32, i64, i32, vp]),
    ("cbm_plan_workspace_bytes", i64, [vp, i32, i64, i32, i32, i32]),
    ("cbm_matmul", C.c_int, [vp, i32, vp, i32, i64, vp, i32, i64, i64, vp, i64, vp]),
    ("cbm_matmul_adjoint", C.c_int, [vp, i32, vp, i32, i64, vp, i32, i64, i64, vp, i64, vp]),
    ("cbm_matmul_host", C.c_int, [vp, i32, vp, i32, i64, vp, i32, i64, i64, i64, vp, vp, vp, i64, vp]),
    ("cbm_matmul_gin", C.c_int, [vp, C.c_float, vp, i32, i64, vp, i32, i64, i64, vp, i64, vp]),
    ("cbm_plan_prepare_adjoint", C.c_int, [vp, vp]),
    ("cbm_plan_set_timeout", C.c_int, [vp, i64]),
    ("cbm_plan_set_passes", C.c_int, [vp, i32]),
    ("cbm_plan_set_host_overlap", C.c_int, [vp, i32]),
    ("cbm_plan_host_wait", C.c_int, [vp, vp]),
    ("cbm_plan_set_compensation", C.c_int, [vp, i32]),
    ("cbm_plan_debug_set_parent", C.c_int, [vp, i64, i32, vp]),
    ("cbm_plan_debug_check_transpose", C.c_int, [vp, vp]),
    ("cbm_plan_error", C.c_int, [vp, vp, C.POINTER(i32), C.POINTER(i64)]),
    ("cbm_matmul_noalloc", C.c_int, [vp, vp, vp, i64, i64, vp, vp, i64, vp, vp, vp, i64, vp, vp]),
    ("cbm_direct_workspace_bytes", i64, [i64]),
    ("cbm_direct_status", C.c_int, [vp, vp, C.POINTER(i32), C.POINTER(i64)]),
    ("cbm_s_spmm_csr_int32", C.c_int, [vp, vp, vp, vp, i64, i64, i64, vp, i64, vp, vp, i64, vp]),
    ("cbm_s_spmm_csr_t_int32", C.c_int, [vp, vp, vp, vp, i64, i64, i64, vp, i64, vp, vp, i64, vp]),
    ("cbm_s_spmm_add_csr_int32", C.c_int, [vp, vp, vp, vp, i64, i64, i64, vp, i64, C.c_float, vp, vp, i64, vp]),
    ("cbm_s_spmm_update_csr_int32", C.c_int, [vp, vp, vp, vp, i64, i64, i64, vp, i64, vp, i64, vp, vp, i64, vp,
                                              vp, i64, vp]),
    ("cbm_s_spmm_fused_update_csr_int32", C.c_int, [vp, vp, vp, vp, i64, i64, i64, vp, i64, vp, i64, vp, vp, i64,
                                                    vp, vp, vp, i64, vp]),
    ("cbm_s_spmm_update_add_csr_int32", C.c_int, [vp, vp, vp, vp, i64, i64, i64, vp, i64, C.c_float, vp, i64, vp,
                                                  vp, i64, vp, vp, i64, vp]),
    ("cbm_s_update_csr_int32", C.c_int, [vp, i64, vp, vp, i64, vp, i64, i64, vp, i64, vp]),
    ("cbm_s_fused_update_csr_int32", C.c_int, [vp, i64, vp, vp, i64, vp, vp, i64, i64, vp, i64, vp]),
    ("cbm_plan_stat", i64, [vp, i32]),
    ("cbm_plan_destroy", None, [vp]),
    ("cbm_status_string", C.c_char_p, [i32]),
]

_lib = None


def load():
    """Loads the library once; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m cbm._build`")
    lib = C.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def status_string(code):
    return load().cbm_status_string(int(code)).decode()


class CbmError(RuntimeError):
    """A non-zero status from the C ABI (a RuntimeError, like the reference's TORCH_CHECK)."""

    def __init__(self, code, what):
        super().__init__(f"{what}: {status_string(code)} (status {code})")
        self.code = code


def check(code, what):
    if code != OK:
        raise CbmError(code, what)
