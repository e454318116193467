"""Batched solve of many small independent systems (cfd_batch_*).

The 1-D network solver of CFDrs solves one Kirchhoff system per design
candidate (``LinearSystemSolver::solve_with_initial_guess``,
``crates/cfd-1d/src/solver/core/linear_system.rs:114-155``, called per
candidate from ``crates/cfd-optim/src/metrics/blueprint_graph.rs:48-135``).
:class:`NetworkBatch` solves all of them in one device call: Jacobi-PCG per
system with the reference's row-equilibrated residual test.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .device import Context, context
from .krylov import IterativeSolverConfig, Precision, SolveError, Termination
from .sparse import CsrMatrix


@dataclass
class BatchReport:
    num_systems: int
    converged_systems: int
    total_iterations: int
    max_iterations: int
    max_rel_residual: float
    device_ms: float
    termination: np.ndarray
    iterations: np.ndarray
    rel_residual: np.ndarray


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class NetworkBatch:
    """A set of square systems resident on the device (``cfd_batch``)."""

    def __init__(self, systems: list[CsrMatrix], ctx: Context | None = None):
        self.ctx = ctx or context()
        sizes = np.array([m.nrows for m in systems], dtype=np.int64)
        self.sys_row = np.zeros(len(systems) + 1, dtype=np.int64)
        np.cumsum(sizes, out=self.sys_row[1:])
        nnz = np.array([m.nnz for m in systems], dtype=np.int64)
        nnz_off = np.zeros(len(systems) + 1, dtype=np.int64)
        np.cumsum(nnz, out=nnz_off[1:])
        self.row_ptr = np.empty(self.sys_row[-1] + 1, dtype=np.int64)
        self.row_ptr[-1] = nnz_off[-1]
        for s, m in enumerate(systems):
            if m.nrows != m.ncols:
                raise SolveError(f"system {s} is not square")
            self.row_ptr[self.sys_row[s]:self.sys_row[s + 1]] = m.row_ptr[:-1] + nnz_off[s]
        self.col = np.concatenate([m.col for m in systems]).astype(np.int32) if systems else np.zeros(0, np.int32)
        self.val = np.concatenate([m.val for m in systems]) if systems else np.zeros(0)
        self.num_systems = len(systems)
        self.rows = int(self.sys_row[-1])
        h = C.c_void_p()
        _lib.check(_lib.load().cfd_batch_create(self.ctx.h, self.num_systems, _p(self.sys_row), _p(self.row_ptr),
                                                _p(self.col), _p(self.val), C.byref(h)))
        self.h = h

    def split(self, v: np.ndarray) -> list[np.ndarray]:
        return [v[self.sys_row[s]:self.sys_row[s + 1]] for s in range(self.num_systems)]

    def update_values(self, val) -> None:
        v = np.ascontiguousarray(val, dtype=np.float64)
        if v.shape[0] != self.val.shape[0]:
            raise SolveError("value array must match the batch's nonzeros")
        _lib.check(_lib.load().cfd_batch_update_values(self.h, _p(v)))
        self.val = v

    def solve(self, b, x=None, config: IterativeSolverConfig | None = None,
              precision: Precision = Precision.FP64, inner_tolerance: float = 1e-4,
              max_outer: int = 20) -> tuple[np.ndarray, BatchReport]:
        """Solve every system; b and x are concatenated over the systems (host)."""
        cfg = (config or IterativeSolverConfig(0.0, 1e-10, 20000)).to_c()
        bb = np.ascontiguousarray(b, dtype=np.float64)
        if bb.shape[0] != self.rows:
            raise SolveError(f"rhs has {bb.shape[0]} entries, the batch {self.rows} rows")
        xx = np.zeros(self.rows) if x is None else np.array(x, dtype=np.float64, copy=True)
        opt = _lib.SolveOptionsC(0, 1, int(precision), 0, inner_tolerance, max_outer, 0)
        term = np.zeros(self.num_systems, np.int32)
        its = np.zeros(self.num_systems, np.int32)
        res = np.zeros(self.num_systems, np.float64)
        rep = _lib.BatchReportC()
        st = _lib.load().cfd_batch_solve(self.h, C.byref(opt), _p(bb), _p(xx), C.byref(cfg), _p(term), _p(its),
                                         _p(res), C.byref(rep))
        if st != _lib.CFD_OK:
            raise SolveError(f"batched solve failed: {_lib.STATUS_NAMES.get(st, st)}: "
                             f"{_lib.load().cfd_last_error().decode()}")
        return xx, BatchReport(rep.num_systems, rep.converged_systems, rep.total_iterations, rep.max_iterations,
                               rep.max_rel_residual, rep.device_ms, term, its, res)

    def autotune(self, precision: Precision = Precision.FP64, sample_iterations: int = 64) -> dict:
        _lib.check(_lib.load().cfd_batch_autotune(self.h, int(precision), sample_iterations))
        return self.config(precision)

    def config(self, precision: Precision = Precision.FP64) -> dict:
        rows = np.zeros(4, np.int32)
        thr = np.zeros(4, np.int32)
        sysn = np.zeros(4, np.int32)
        _lib.check(_lib.load().cfd_batch_config(self.h, int(precision), _p(rows), _p(thr), _p(sysn)))
        return {"bucket_rows": rows.tolist(), "threads": thr.tolist(), "systems": sysn.tolist()}

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            try:
                _lib.load().cfd_batch_destroy(h)
            except Exception:
                pass
            self.h = None


__all__ = ["NetworkBatch", "BatchReport", "Termination"]
