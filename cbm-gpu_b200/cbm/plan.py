"""Device plan: a CBM structure uploaded in the fused kernel's layout.

Thin owner of a ``cbm_plan*`` (include/cbm_b200.h).  The product path is the
CUDA library only: there is no CPU fallback; if the library is missing or the
tensors are not on the plan's GPU, calls raise RuntimeError.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib

_DT = {torch.float32: _lib.F32, torch.bfloat16: _lib.BF16}
OPS = {"ax": _lib.OP_AX, "adx": _lib.OP_ADX, "dadx": _lib.OP_DADX,
       "values_add": _lib.OP_VALUES_ADD, "values_ratio": _lib.OP_VALUES_RATIO, "dad_add": _lib.OP_DAD_ADD}


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, torch.Tensor):
        return a.data_ptr() if a.numel() else None
    return a.ctypes.data if a.size else None


def _stream(device):
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


class Plan:
    """Owns the device layout of one CBM matrix and runs its products."""

    def __init__(self, row_ptr, col_idx, values, n_rows, n_cols, branches, src, dst, multipliers=None,
                 host=False):
        self._lib = _lib.load()
        self._h = None
        if not torch.cuda.is_available():
            raise RuntimeError("CBM products need a CUDA device")
        self.device = torch.device("cuda", torch.cuda.current_device())
        keep = []

        def arr(a, dt, name):
            if a is None:
                return None
            if host:
                a = np.ascontiguousarray(a.cpu().numpy() if isinstance(a, torch.Tensor) else a, dtype=dt)
            else:
                if not isinstance(a, torch.Tensor) or not a.is_cuda:
                    raise RuntimeError(f"{name}: tensor is not a CUDA tensor")
                tdt = torch.int32 if dt == np.int32 else torch.float32
                if a.dtype != tdt:
                    raise RuntimeError(f"{name}: expected dtype {tdt}, got {a.dtype}")
                a = a.contiguous()
            keep.append(a)
            return a

        rp = arr(row_ptr, np.int32, "row_ptr")
        ci = arr(col_idx, np.int32, "col_idx")
        va = arr(values, np.float32, "values")
        br = arr(branches, np.int32, "mca_branches")
        s = arr(src, np.int32, "mca_src_node_idx")
        d = arr(dst, np.int32, "mca_dst_node_idx")
        m = arr(multipliers, np.float32, "multipliers") if multipliers is not None and len(multipliers) else None
        n_rows, n_cols = int(n_rows), int(n_cols)
        nnz = int(ci.shape[0]) if ci is not None else 0
        h = C.c_void_p()
        rc = self._lib.cbm_plan_create(
            _ptr(rp), _ptr(ci), _ptr(va), n_rows, n_cols, nnz, _ptr(br), int(br.shape[0]) if br is not None else 0,
            _ptr(s), _ptr(d), int(s.shape[0]) if s is not None else 0, _ptr(m),
            _lib.INPUT_HOST if host else _lib.INPUT_DEVICE, _stream(self.device), C.byref(h))
        _lib.check(rc, "cbm_plan_create")
        self._h = h
        self.n_rows, self.n_cols, self.nnz = n_rows, n_cols, nnz
        self._ws = {}

    # ---- housekeeping -------------------------------------------------------
    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h is not None and h.value:
            try:
                self._lib.cbm_plan_destroy(h)
            except Exception:  # interpreter shutdown
                pass

    def stat(self, which):
        return int(self._lib.cbm_plan_stat(self._h, which))

    @property
    def stats(self):
        names = ["rows", "cols", "nnz", "edges", "branches", "levels", "internal", "chunks", "long_rows",
                 "unit_values", "grid", "launches"]
        return {n: self.stat(i) for i, n in enumerate(names)}

    def set_multipliers(self, d):
        if not (isinstance(d, torch.Tensor) and d.is_cuda and d.dtype == torch.float32 and d.numel() == self.n_rows):
            raise RuntimeError("multipliers must be a CUDA float32 tensor with one entry per row")
        d = d.contiguous()
        _lib.check(self._lib.cbm_plan_set_multipliers(self._h, d.data_ptr(), _stream(self.device)),
                   "cbm_plan_set_multipliers")
        torch.cuda.current_stream(self.device).synchronize()

    def tune(self, chunk_nnz=256, rows_per_claim=4, variant="auto", hot_rows=65536, team=0, rows_per_claim_deep=0):
        v = {"auto": _lib.VARIANT_AUTO, "register": _lib.VARIANT_REGISTER, "staged": _lib.VARIANT_STAGED,
             "tma": _lib.VARIANT_TMA}[variant]
        _lib.check(self._lib.cbm_plan_tune(self._h, int(chunk_nnz), int(rows_per_claim), int(rows_per_claim_deep), v,
                                           int(hot_rows), int(team), _stream(self.device)), "cbm_plan_tune")
        self._ws.clear()

    def set_compensation(self, min_depth):
        """BF16 X: compensated propagation from tree depth ``min_depth`` on (-1: off)."""
        _lib.check(self._lib.cbm_plan_set_compensation(self._h, int(min_depth)), "cbm_plan_set_compensation")
        self._ws.clear()

    def set_passes(self, passes):
        """'auto', 'fused' or 'two': one fused pass, or a delta pass then a
        propagation pass (FP32 Y); bit-identical results."""
        v = {"auto": _lib.PASSES_AUTO, "fused": _lib.PASSES_FUSED, "two": _lib.PASSES_TWO}[passes]
        _lib.check(self._lib.cbm_plan_set_passes(self._h, v), "cbm_plan_set_passes")

    def set_timeout(self, ns):
        _lib.check(self._lib.cbm_plan_set_timeout(self._h, int(ns)), "cbm_plan_set_timeout")

    def prepare_adjoint(self):
        _lib.check(self._lib.cbm_plan_prepare_adjoint(self._h, _stream(self.device)), "cbm_plan_prepare_adjoint")
        self._ws = {k: v for k, v in self._ws.items() if not k[-1]}

    def error(self):
        """Synchronises and returns (device status, info); clears the status."""
        st = C.c_int32(0)
        info = C.c_int64(0)
        _lib.check(self._lib.cbm_plan_error(self._h, _stream(self.device), C.byref(st), C.byref(info)),
                   "cbm_plan_error")
        return int(st.value), int(info.value)

    def check_device(self):
        st, info = self.error()
        if st != _lib.OK:
            raise _lib.CbmError(st, f"device-side error (info {info})")

    # ---- products -------------------------------------------------------------
    def workspace(self, op, cols, xdt, ydt, adjoint):
        key = (op, cols, xdt, ydt, adjoint)
        ws = self._ws.get(key)
        if ws is None:
            nbytes = int(self._lib.cbm_plan_workspace_bytes(self._h, op, cols, xdt, ydt, int(adjoint)))
            ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.device)
            self._ws[key] = ws
        return ws

    def _operand(self, t, rows, name):
        if not isinstance(t, torch.Tensor) or not t.is_cuda:
            raise RuntimeError(f"{name}: tensor is not a CUDA tensor")
        if t.device != self.device:
            raise RuntimeError(f"{name}: tensor is on {t.device}, the plan on {self.device}")
        if t.dtype not in _DT:
            raise RuntimeError(f"{name}: dtype {t.dtype} is not supported (float32 or bfloat16)")
        if t.dim() != 2 or t.shape[0] != rows:
            raise RuntimeError(f"{name}: expected shape [{rows}, C], got {list(t.shape)}")
        if t.shape[1] > 1 and t.stride(1) != 1:
            raise RuntimeError(f"{name}: rows must be contiguous (stride(1) == 1)")
        return _DT[t.dtype], max(int(t.stride(0)), int(t.shape[1]), 1)

    def matmul(self, op, x, y):
        """y <- op(A) x on the current stream (no synchronisation)."""
        op = OPS[op] if isinstance(op, str) else int(op)
        xdt, ldx = self._operand(x, self.n_cols, "rhs")
        ydt, ldy = self._operand(y, self.n_rows, "res")
        if x.shape[1] != y.shape[1]:
            raise RuntimeError(f"rhs has {x.shape[1]} columns, res {y.shape[1]}")
        cols = int(x.shape[1])
        ws = self.workspace(op, cols, xdt, ydt, False)
        rc = self._lib.cbm_matmul(self._h, op, x.data_ptr(), xdt, ldx, y.data_ptr(), ydt, ldy, cols,
                                  ws.data_ptr(), ws.numel(), _stream(self.device))
        _lib.check(rc, "cbm_matmul")

    def matmul_gin(self, x, y, epsilon):
        """y <- A x + (1 + epsilon) x (GIN aggregation) on the current stream."""
        xdt, ldx = self._operand(x, self.n_cols, "rhs")
        ydt, ldy = self._operand(y, self.n_rows, "res")
        if x.shape[1] != y.shape[1]:
            raise RuntimeError(f"rhs has {x.shape[1]} columns, res {y.shape[1]}")
        cols = int(x.shape[1])
        ws = self.workspace(_lib.OP_GIN, cols, xdt, ydt, False)
        rc = self._lib.cbm_matmul_gin(self._h, float(epsilon), x.data_ptr(), xdt, ldx, y.data_ptr(), ydt, ldy, cols,
                                      ws.data_ptr(), ws.numel(), _stream(self.device))
        _lib.check(rc, "cbm_matmul_gin")

    def matmul_host(self, op, x, y, slab_cols=64, overlap_calls=False):
        """y <- op(A) x with x and y in host memory (pinned for full-speed copies):
        column slabs are copied in, multiplied and copied out on overlapping
        streams.  Device buffers of the operand shapes are allocated on the first
        call and reused.  Returns once queued; the current stream waits for the
        last copy (synchronise it before reading y).  overlap_calls: this call's
        copy-in may run under the previous call's copy-out (x must then be
        complete in host memory when the call is made), and the current stream
        waits only for this call's products: call host_wait() before
        synchronising to read y (see cbm_plan_set_host_overlap)."""
        op = OPS[op] if isinstance(op, str) else int(op)
        for t, rows, name in ((x, self.n_cols, "rhs"), (y, self.n_rows, "res")):
            if not isinstance(t, torch.Tensor) or t.is_cuda:
                raise RuntimeError(f"{name}: expected a host (CPU) tensor")
            if t.dtype not in _DT:
                raise RuntimeError(f"{name}: dtype {t.dtype} is not supported (float32 or bfloat16)")
            if t.dim() != 2 or t.shape[0] != rows or (t.shape[1] > 1 and t.stride(1) != 1):
                raise RuntimeError(f"{name}: expected a row-major [{rows}, C] tensor")
        if x.shape[1] != y.shape[1]:
            raise RuntimeError(f"rhs has {x.shape[1]} columns, res {y.shape[1]}")
        cols = int(x.shape[1])
        xdt, ydt = _DT[x.dtype], _DT[y.dtype]
        key = (cols, x.dtype, y.dtype)
        bufs = getattr(self, "_host_bufs", {})
        if key not in bufs:
            if bufs:
                # copies of earlier calls may still use the old buffers
                self.host_wait()
                torch.cuda.current_stream(self.device).synchronize()
            bufs.clear()
            bufs[key] = (torch.empty(self.n_cols, cols, dtype=x.dtype, device=self.device),
                         torch.empty(self.n_rows, cols, dtype=y.dtype, device=self.device))
            self._host_bufs = bufs
        xd, yd = bufs[key]
        ws = self.workspace(op, cols, xdt, ydt, False)  # covers every slab width
        _lib.check(self._lib.cbm_plan_set_host_overlap(self._h, 1 if overlap_calls else 0),
                   "cbm_plan_set_host_overlap")
        rc = self._lib.cbm_matmul_host(self._h, op, x.data_ptr(), xdt, max(int(x.stride(0)), cols, 1), y.data_ptr(),
                                       ydt, max(int(y.stride(0)), cols, 1), cols, int(slab_cols), xd.data_ptr(),
                                       yd.data_ptr(), ws.data_ptr(), ws.numel(), _stream(self.device))
        _lib.check(rc, "cbm_matmul_host")

    def host_wait(self):
        """The current stream waits for every copy-out of matmul_host calls
        made so far (needed after overlap_calls before y is read)."""
        _lib.check(self._lib.cbm_plan_host_wait(self._h, _stream(self.device)), "cbm_plan_host_wait")

    def adjoint(self, op, g, dx):
        """dx <- op(A)^T g on the current stream."""
        op = OPS[op] if isinstance(op, str) else int(op)
        gdt, ldg = self._operand(g, self.n_rows, "grad")
        ddt, lddx = self._operand(dx, self.n_cols, "grad_input")
        if g.shape[1] != dx.shape[1]:
            raise RuntimeError(f"grad has {g.shape[1]} columns, grad_input {dx.shape[1]}")
        cols = int(g.shape[1])
        if not self.stat(_lib.P_CHUNKS) >= 0:
            raise RuntimeError("invalid plan")
        self.prepare_adjoint() if not getattr(self, "_adj_ready", False) else None
        self._adj_ready = True
        ws = self.workspace(op, cols, gdt, ddt, True)
        rc = self._lib.cbm_matmul_adjoint(self._h, op, g.data_ptr(), gdt, ldg, dx.data_ptr(), ddt, lddx, cols,
                                          ws.data_ptr(), ws.numel(), _stream(self.device))
        _lib.check(rc, "cbm_matmul_adjoint")
