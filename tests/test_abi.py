"""The C ABI: the library loads, exports every function include/cbm_b200.h
declares, and rejects bad structures on the host (no GPU needed)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import REPO, near_dup_graph


def _declared_functions():
    text = open(os.path.join(REPO, "include", "cbm_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w\*\s]+?\b(cbm_\w+)\s*\(", text, flags=re.M)))


def test_every_declared_function_is_exported(lib):
    names = _declared_functions()
    assert len(names) >= 18
    for name in names:
        assert hasattr(lib, name), name


def test_python_binding_covers_the_header():
    from cbm import _lib

    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert set(_declared_functions()) == bound


def test_status_strings(lib):
    from cbm import _lib

    for code in range(13):
        assert _lib.status_string(code)
    assert "timed out" in _lib.status_string(_lib.ERR_TIMEOUT)


def _validate(lib, rp, ci, n_rows, n_cols, br, src, dst):
    a = [np.ascontiguousarray(v, dtype=np.int32) for v in (rp, ci, br, src, dst)]
    return lib.cbm_validate(a[0].ctypes.data, a[1].ctypes.data if a[1].size else None, n_rows, n_cols, a[1].size,
                            a[2].ctypes.data if a[2].size else None, a[2].size,
                            a[3].ctypes.data if a[3].size else None, a[4].ctypes.data if a[4].size else None,
                            a[3].size)


@pytest.fixture(scope="module")
def structure():
    from cbm import cbm_mkl_cpp

    ei = near_dup_graph(200, seed=1)
    return cbm_mkl_cpp.build(ei[0], ei[1], 200, 0)


def test_valid_structure_accepted(lib, structure):
    s = structure
    assert _validate(lib, s.csr_ptr, s.csr_col, 200, 200, s.branches, s.src, s.dst) == 0


def test_cycle_rejected(lib, structure):
    from cbm import _lib

    s = structure
    assert s.src.size >= 2
    src, dst = s.src.copy(), s.dst.copy()
    # make the first edge's parent a descendant of its child: u -> v and v -> u
    src = np.concatenate([src, [dst[0]]])
    dst = np.concatenate([dst, [src[0]]])
    br = s.branches.copy()
    br[-1] += 1
    assert _validate(lib, s.csr_ptr, s.csr_col, 200, 200, br, src, dst) in (_lib.ERR_STRUCTURE,)


def test_duplicate_child_rejected(lib, structure):
    from cbm import _lib

    s = structure
    src = np.concatenate([s.src, [s.src[0]]])
    dst = np.concatenate([s.dst, [s.dst[0]]])
    br = s.branches.copy()
    br[-1] += 1
    assert _validate(lib, s.csr_ptr, s.csr_col, 200, 200, br, src, dst) == _lib.ERR_STRUCTURE


def test_out_of_range_rejected(lib, structure):
    from cbm import _lib

    s = structure
    src = s.src.copy()
    src[0] = 200
    assert _validate(lib, s.csr_ptr, s.csr_col, 200, 200, s.branches, src, s.dst) == _lib.ERR_INDEX
    col = s.csr_col.copy()
    col[3] = -1
    assert _validate(lib, s.csr_ptr, col, 200, 200, s.branches, s.src, s.dst) == _lib.ERR_INDEX


def test_bad_offsets_rejected(lib, structure):
    from cbm import _lib

    s = structure
    br = s.branches.copy()
    br[-1] -= 1
    assert _validate(lib, s.csr_ptr, s.csr_col, 200, 200, br, s.src, s.dst) == _lib.ERR_STRUCTURE
    rp = s.csr_ptr.copy()
    rp[5], rp[6] = rp[6], rp[5] + 0
    rp[5] = rp[6] + 1
    assert _validate(lib, rp, s.csr_col, 200, 200, s.branches, s.src, s.dst) == _lib.ERR_STRUCTURE


def test_self_parent_rejected(lib, structure):
    from cbm import _lib

    s = structure
    src = s.src.copy()
    src[0] = s.dst[0]
    assert _validate(lib, s.csr_ptr, s.csr_col, 200, 200, s.branches, src, s.dst) == _lib.ERR_STRUCTURE


def test_plan_needs_cuda_without_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from cbm.plan import Plan

    with pytest.raises(RuntimeError):
        Plan(np.array([0, 0], np.int32), np.array([], np.int32), None, 1, 1, np.array([0], np.int32),
             np.array([], np.int32), np.array([], np.int32), host=True)


def test_null_handle_calls_are_errors(lib):
    from cbm import _lib

    assert lib.cbm_matmul(None, 0, None, 0, 1, None, 0, 1, 1, None, 0, None) == _lib.ERR_INVALID
    assert lib.cbm_plan_stat(None, 0) == -1
    assert lib.cbm_plan_workspace_bytes(None, 0, 4, 0, 0, 0) == -1
    lib.cbm_plan_destroy(None)
    h = C.c_void_p()
    assert lib.cbm_build(None, None, 5, 3, 0, 1, 0, C.byref(h)) == _lib.ERR_INVALID
