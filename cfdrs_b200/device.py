"""Device handles: the CUDA context/stream (``cfd_context``) and device CSR
matrices (``cfd_csr``), with the upload cached per host matrix so repeated
solves on one pattern pay it once (the reference borrows the matrix per call,
``krylov.rs:330``)."""
from __future__ import annotations

import ctypes as C
import threading
import weakref

import numpy as np

from . import _lib
from .sparse import CsrMatrix

_contexts: dict[int, "Context"] = {}
# cudaStreamLegacy: the handle value CUDA reserves for the legacy default stream.
LEGACY_STREAM = 0x1
_ctx_lock = threading.Lock()


class Context:
    """One device and one CUDA stream (``cfd_context``)."""

    def __init__(self, device: int = 0):
        L = _lib.load()
        h = C.c_void_p()
        _lib.check(L.cfd_context_create(device, C.byref(h)))
        self.h = h
        self.device = device

    def set_stream(self, stream_ptr: int | None) -> None:
        """Run this context's work on an existing CUDA stream (e.g. torch's);
        ``None`` returns to the context's own stream. Handle 0 is CUDA's legacy
        default stream (torch's default stream) and is passed on as such."""
        if stream_ptr is None:
            arg = None
        elif stream_ptr == 0:
            arg = LEGACY_STREAM
        else:
            arg = stream_ptr
        _lib.check(_lib.load().cfd_context_set_stream(self.h, C.c_void_p(arg)))

    def synchronize(self) -> None:
        _lib.check(_lib.load().cfd_context_synchronize(self.h))

    def set_cluster_solve(self, enable: bool) -> None:
        """Whole CG / Jacobi-PCG solves of small systems in one thread-block
        cluster launch (the default) or always the multi-kernel solve."""
        _lib.check(_lib.load().cfd_context_set_cluster_solve(self.h, 1 if enable else 0))

    def kernel_stats(self) -> dict:
        s = _lib.KernelStatsC()
        _lib.check(_lib.load().cfd_last_kernel_stats(self.h, C.byref(s)))
        return {"launches": s.launches, "spmv_launches": s.spmv_launches, "spmv_bytes": s.spmv_bytes}

    def close(self) -> None:
        if self.h:
            _lib.load().cfd_context_destroy(self.h)
            self.h = None


def context(device: int = 0) -> Context:
    """The process-wide context of ``device`` (created on first use)."""
    with _ctx_lock:
        ctx = _contexts.get(device)
        if ctx is None:
            ctx = Context(device)
            _contexts[device] = ctx
        return ctx


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class DeviceCsr:
    """A CSR matrix resident on the device (``cfd_csr``)."""

    def __init__(self, m: CsrMatrix, ctx: Context | None = None):
        self.ctx = ctx or context()
        self.shape = m.shape
        self.nnz = m.nnz
        h = C.c_void_p()
        rp = np.ascontiguousarray(m.row_ptr, dtype=np.int64)
        col = np.ascontiguousarray(m.col, dtype=np.int32)
        val = np.ascontiguousarray(m.val, dtype=np.float64)
        _lib.check(_lib.load().cfd_csr_create_i32(self.ctx.h, m.nrows, m.ncols, m.nnz, _ptr(rp), _ptr(col),
                                                  _ptr(val), C.byref(h)))
        self.h = h
        self.version = getattr(m, "version", 0)  # host value version this copy holds

    def update_values(self, values) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        if v.shape[0] != self.nnz:
            raise ValueError("value array must match nnz")
        _lib.check(_lib.load().cfd_csr_update_values(self.h, _ptr(v)))

    def layout(self) -> dict:
        """Device layout of this matrix (row blocks, column codes, x staging)."""
        info = _lib.LayoutInfoC()
        _lib.check(_lib.load().cfd_csr_layout(self.h, C.byref(info)))
        return {f: getattr(info, f) for f, _ in info._fields_}

    PATHS = {"timed": -2, "auto": -1, "split": 0, "record": 1, "x_staged": 2, "sliced": 3, "diagonal": 4}

    def set_path(self, path: str, fp32: bool) -> None:
        """Set the SpMV pipeline of one precision: "auto" (the default rule),
        "timed" (time the eligible pipelines at the next SpMV), or a pipeline."""
        _lib.check(_lib.load().cfd_csr_set_path(self.h, 1 if fp32 else 0, self.PATHS[path]))

    def spmv(self, x_dev_ptr: int, y_dev_ptr: int, fp32: bool = False) -> None:
        """y = A x on device pointers."""
        fn = _lib.load().cfd_spmv_f32 if fp32 else _lib.load().cfd_spmv
        _lib.check(fn(self.h, C.c_void_p(x_dev_ptr), C.c_void_p(y_dev_ptr)))

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            try:
                _lib.load().cfd_csr_destroy(h)
            except Exception:
                pass
            self.h = None


def layout_check(m: CsrMatrix, x: np.ndarray):
    """Host-only walk of the SpMV device layout (``cfd_layout_check``): returns
    y = A x evaluated through the kernels' index arithmetic and the layout
    statistics; raises CfdError if any staged index leaves its region."""
    rp = np.ascontiguousarray(m.row_ptr, dtype=np.int64)
    col = np.ascontiguousarray(m.col, dtype=np.int32)
    val = np.ascontiguousarray(m.val, dtype=np.float64)
    xx = np.ascontiguousarray(x, dtype=np.float64)
    if xx.shape[0] != m.ncols:
        raise ValueError("x must have ncols entries")
    y = np.zeros(m.nrows)
    info = _lib.LayoutInfoC()
    _lib.check(_lib.load().cfd_layout_check(m.nrows, m.ncols, m.nnz, _ptr(rp), _ptr(col), _ptr(val), _ptr(xx),
                                            _ptr(y), C.byref(info)))
    return y, {f: getattr(info, f) for f, _ in info._fields_}


_uploads: "weakref.WeakKeyDictionary[CsrMatrix, DeviceCsr]" = weakref.WeakKeyDictionary()


def device_matrix(m, ctx: Context | None = None) -> DeviceCsr:
    """Upload ``m`` once and reuse the device copy while ``m`` is alive; values
    changed since the upload (``CsrMatrix.set_values``) are copied to the
    device first, with the pattern's layout kept."""
    if isinstance(m, DeviceCsr):
        return m
    d = _uploads.get(m)
    if d is None or (ctx is not None and d.ctx is not ctx):
        d = DeviceCsr(m, ctx)
        _uploads[m] = d
    elif d.version != getattr(m, "version", 0):
        d.update_values(m.val)
        d.version = m.version
    return d


def mark_synced(m, d: DeviceCsr) -> None:
    """Record that ``d`` already holds ``m``'s current values (written on the
    device by the caller), so no upload follows."""
    d.version = m.version


def refresh_device_values(m) -> None:
    """Copy ``m``'s current values to its device copy, if it has one."""
    d = _uploads.get(m) if isinstance(m, CsrMatrix) else None
    if d is not None:
        d.update_values(m.val)
        d.version = m.version
