"""Batched solve of many small independent systems (cfd_batch_*).

The 1-D network solver of CFDrs solves one Kirchhoff system per design
candidate (``LinearSystemSolver::solve_with_initial_guess``,
``crates/cfd-1d/src/solver/core/linear_system.rs:114-155``, called per
candidate from ``crates/cfd-optim/src/metrics/blueprint_graph.rs:48-135``).
:class:`NetworkBatch` solves all of them in one device call: the solver's
full cascade (:meth:`NetworkBatch.solve_linear_systems`), or Jacobi-PCG per
system with the reference's row-equilibrated residual test
(:meth:`NetworkBatch.solve`).
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


LS_CG, LS_BICGSTAB, LS_DETECT = 0, 1, 2
LS_PATHS = ["krylov", "direct", "direct_unscaled", "krylov_fallback", "failed", "error"]


@dataclass
class LinearSystemReport:
    """Per batch and per system outcome of :meth:`NetworkBatch.solve_linear_systems`:
    ``method`` (LS_CG / LS_BICGSTAB), ``path`` (an index into LS_PATHS),
    ``termination`` of the Krylov solve (-1 when none ran), its ``iterations``
    and ``residual`` = ||D (A x - b)|| / ||D b|| of the returned solution."""
    num_systems: int
    solved_systems: int
    total_iterations: int
    max_iterations: int
    max_residual: float
    device_ms: float
    method: np.ndarray
    path: np.ndarray
    termination: np.ndarray
    iterations: np.ndarray
    residual: np.ndarray
    phase_ms: dict = None  # device time of the direct, Krylov and fallback phases


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


@dataclass
class PackedNetworks:
    """Networks concatenated as cfd_batch_create_networks takes them: node and
    edge offsets per network, edge endpoints local to their network, and the
    Dirichlet mask and pressures per global node."""
    node_off: np.ndarray
    edge_off: np.ndarray
    edge_i: np.ndarray
    edge_j: np.ndarray
    fixed: np.ndarray
    fixed_value: np.ndarray
    conductance: np.ndarray

    @property
    def num_systems(self) -> int:
        return self.node_off.shape[0] - 1

    @property
    def rows(self) -> int:
        return int(self.node_off[-1])

    @property
    def edges(self) -> int:
        return int(self.edge_off[-1])


def pack_networks(networks) -> PackedNetworks:
    """From objects with ``n_nodes, edges_i, edges_j, conductance, fixed,
    fixed_value`` (``problems.Network``)."""
    nodes = np.array([int(n.n_nodes) for n in networks], dtype=np.int64)
    edges = np.array([len(n.edges_i) for n in networks], dtype=np.int64)
    node_off = np.concatenate([[0], np.cumsum(nodes)]).astype(np.int64)
    edge_off = np.concatenate([[0], np.cumsum(edges)]).astype(np.int64)

    def cat(name, dtype):
        parts = [np.asarray(getattr(n, name), dtype=dtype) for n in networks]
        return np.ascontiguousarray(np.concatenate(parts) if parts else np.zeros(0, dtype))
    return PackedNetworks(node_off, edge_off, cat("edges_i", np.int32), cat("edges_j", np.int32),
                          cat("fixed", np.int8), cat("fixed_value", np.float64), cat("conductance", np.float64))


def network_assemble_host(packed: PackedNetworks, conductance=None, neumann=None):
    """The device assembly's pattern and values computed on the host by the
    same code (``cfd_network_assemble_host``). Returns ``(row_ptr, col, val,
    rhs)``; ``val`` and ``rhs`` are None without conductances."""
    L = _lib.load()
    nnz = C.c_int64()
    args = (packed.num_systems, _p(packed.node_off), _p(packed.edge_off), _p(packed.edge_i), _p(packed.edge_j),
            _p(packed.fixed), _p(packed.fixed_value))
    _lib.check(L.cfd_network_assemble_host(*args, None, None, C.byref(nnz), None, None, None, None))
    rp = np.zeros(packed.rows + 1, np.int64)
    col = np.zeros(nnz.value, np.int32)
    g = None if conductance is None else np.ascontiguousarray(conductance, dtype=np.float64)
    q = None if neumann is None else np.ascontiguousarray(neumann, dtype=np.float64)
    val = None if g is None else np.zeros(nnz.value)
    rhs = None if g is None else np.zeros(packed.rows)
    _lib.check(L.cfd_network_assemble_host(*args, _p(g), _p(q), C.byref(nnz), _p(rp), _p(col), _p(val), _p(rhs)))
    return rp, col, val, rhs


def _torch_cuda(a) -> bool:
    try:
        import torch
    except ImportError:
        return False
    return isinstance(a, torch.Tensor) and a.is_cuda


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

    @classmethod
    def from_networks(cls, networks, ctx: Context | None = None) -> "NetworkBatch":
        """A batch of pipe networks given as edges (``problems.Network``); the
        matrices are assembled on the device by :meth:`assemble`
        (``cfd_batch_create_networks``). The networks' own conductances are
        kept in ``packed.conductance`` but not assembled."""
        self = cls.__new__(cls)
        self.ctx = ctx or context()
        self.packed = pk = pack_networks(networks)
        h = C.c_void_p()
        _lib.check(_lib.load().cfd_batch_create_networks(self.ctx.h, pk.num_systems, _p(pk.node_off),
                                                         _p(pk.edge_off), _p(pk.edge_i), _p(pk.edge_j),
                                                         _p(pk.fixed), _p(pk.fixed_value), C.byref(h)))
        self.h = h
        self.sys_row = pk.node_off
        self.row_ptr, self.col, _, _ = network_assemble_host(pk)
        self.val = np.zeros(self.col.shape[0])
        self.num_systems = pk.num_systems
        self.rows = pk.rows
        return self

    def assemble(self, conductance, neumann=None) -> None:
        """Values and right-hand sides from per-edge conductances (and
        optional per-node Neumann sources), both numpy arrays (host) or both
        float64 CUDA tensors (device, read on torch's current stream)."""
        pk = getattr(self, "packed", None)
        if pk is None:
            raise SolveError("assemble needs a batch made by NetworkBatch.from_networks")
        L = _lib.load()
        if _torch_cuda(conductance):
            import torch
            if conductance.dtype != torch.float64 or conductance.numel() != pk.edges or not conductance.is_contiguous():
                raise SolveError("conductance must be a contiguous float64 tensor with one entry per edge")
            if neumann is not None and (not _torch_cuda(neumann) or neumann.dtype != torch.float64
                                        or neumann.numel() != pk.rows or not neumann.is_contiguous()):
                raise SolveError("neumann must be a contiguous float64 CUDA tensor with one entry per node")
            self.ctx.set_stream(torch.cuda.current_stream(conductance.device).cuda_stream)
            try:
                st = L.cfd_batch_assemble(self.h, C.c_void_p(conductance.data_ptr()),
                                          None if neumann is None else C.c_void_p(neumann.data_ptr()), 1)
            finally:
                self.ctx.set_stream(None)
        else:
            g = np.ascontiguousarray(conductance, dtype=np.float64)
            q = None if neumann is None else np.ascontiguousarray(neumann, dtype=np.float64)
            if g.shape[0] != pk.edges or (q is not None and q.shape[0] != pk.rows):
                raise SolveError(f"need {pk.edges} conductances and {pk.rows} Neumann sources")
            st = L.cfd_batch_assemble(self.h, _p(g), _p(q), 0)
        _lib.check(st)

    def values(self) -> tuple[np.ndarray, np.ndarray]:
        """The batch's current values and right-hand sides (host copies)."""
        val = np.zeros(self.col.shape[0])
        rhs = np.zeros(self.rows)
        _lib.check(_lib.load().cfd_batch_values(self.h, _p(val), _p(rhs)))
        return val, rhs

    def split(self, v: np.ndarray) -> list[np.ndarray]:
        return [v[self.sys_row[s]:self.sys_row[s + 1]] for s in range(self.num_systems)]

    def update_values(self, val) -> None:
        v = np.ascontiguousarray(val, dtype=np.float64)
        if v.shape[0] != self.val.shape[0]:
            raise SolveError("value array must match the batch's nonzeros")
        _lib.check(_lib.load().cfd_batch_update_values(self.h, _p(v)))
        self.val = v

    def solve(self, b=None, x=None, config: IterativeSolverConfig | None = None,
              precision: Precision = Precision.FP64, inner_tolerance: float = 1e-4,
              max_outer: int = 20) -> tuple[np.ndarray, BatchReport]:
        """Solve every system; b and x are concatenated over the systems.
        Host arrays, or float64 CUDA tensors (x then holds the initial guess
        and is overwritten with the solution, on torch's current stream).
        b = None solves with the right-hand sides of the last
        :meth:`assemble`."""
        cfg = (config or IterativeSolverConfig(0.0, 1e-10, 20000)).to_c()
        device = _torch_cuda(x)
        if device:
            import torch
            if x.dtype != torch.float64 or x.numel() != self.rows or not x.is_contiguous():
                raise SolveError("x must be a contiguous float64 CUDA tensor with one entry per row")
            if b is not None and (not _torch_cuda(b) or b.dtype != torch.float64 or b.numel() != self.rows
                                  or not b.is_contiguous()):
                raise SolveError("with a CUDA x, b must be None or a matching contiguous float64 CUDA tensor")
            xx, bp, xp = x, (None if b is None else C.c_void_p(b.data_ptr())), C.c_void_p(x.data_ptr())
        else:
            if _torch_cuda(b):
                raise SolveError("b is a CUDA tensor: pass x as a float64 CUDA tensor as well (device solve)")
            bb = None if b is None else np.ascontiguousarray(b, dtype=np.float64)
            if bb is not None and bb.shape[0] != self.rows:
                raise SolveError(f"rhs has {bb.shape[0]} entries, the batch {self.rows} rows")
            xx = np.zeros(self.rows) if x is None else np.array(x, dtype=np.float64, copy=True)
            bp, xp = _p(bb), _p(xx)
        opt = _lib.SolveOptionsC(0, 1, int(precision), 1 if device else 0, inner_tolerance, max_outer, 0)
        term = np.zeros(self.num_systems, np.int32)
        its = np.zeros(self.num_systems, np.int32)
        res = np.zeros(self.num_systems, np.float64)
        rep = _lib.BatchReportC()
        if device:
            self.ctx.set_stream(torch.cuda.current_stream(x.device).cuda_stream)
        try:
            st = _lib.load().cfd_batch_solve(self.h, C.byref(opt), bp, xp, C.byref(cfg), _p(term), _p(its),
                                             _p(res), C.byref(rep))
        finally:
            if device:
                self.ctx.set_stream(None)
        if st != _lib.CFD_OK:
            raise SolveError(f"batched solve failed: {_lib.STATUS_NAMES.get(st, st)}: "
                             f"{_lib.load().cfd_last_error().decode()}")
        return xx, BatchReport(rep.num_systems, rep.converged_systems, rep.total_iterations, rep.max_iterations,
                               rep.max_rel_residual, rep.device_ms, term, its, res)

    def solve_linear_systems(self, b=None, x=None, tolerance: float = 1e-6, max_iterations: int = 1000,
                             method: int = LS_DETECT, precision: Precision = Precision.FP64,
                             inner_tolerance: float = 1e-4, max_outer: int = 40):
        """``LinearSystemSolver::new().with_method(..).with_tolerance(..)
        .with_max_iterations(..).solve_with_initial_guess`` for every system
        (``cfd_batch_linear_system_solve``): equilibration, dense LU for n <=
        256, CG or BiCGSTAB (``method``: LS_CG, LS_BICGSTAB, or LS_DETECT for
        ``NetworkSolver::detect_solver_method``) with the residual recheck and
        the dense fallback for larger systems. b and x as for :meth:`solve`.
        Returns ``(x, LinearSystemReport)``."""
        device = _torch_cuda(x)
        if device:
            import torch
            if x.dtype != torch.float64 or x.numel() != self.rows or not x.is_contiguous():
                raise SolveError("x must be a contiguous float64 CUDA tensor with one entry per row")
            if b is not None and (not _torch_cuda(b) or b.dtype != torch.float64 or b.numel() != self.rows
                                  or not b.is_contiguous()):
                raise SolveError("with a CUDA x, b must be None or a matching contiguous float64 CUDA tensor")
            xx, bp, xp = x, (None if b is None else C.c_void_p(b.data_ptr())), C.c_void_p(x.data_ptr())
        else:
            if _torch_cuda(b):
                raise SolveError("b is a CUDA tensor: pass x as a float64 CUDA tensor as well (device solve)")
            bb = None if b is None else np.ascontiguousarray(b, dtype=np.float64)
            if bb is not None and bb.shape[0] != self.rows:
                raise SolveError(f"rhs has {bb.shape[0]} entries, the batch {self.rows} rows")
            xx = np.zeros(self.rows) if x is None else np.array(x, dtype=np.float64, copy=True)
            bp, xp = _p(bb), _p(xx)
        opt = _lib.LsOptionsC(tolerance, max_iterations, method, int(precision), 1 if device else 0, max_outer,
                              inner_tolerance)
        res = (_lib.LsResultC * max(self.num_systems, 1))()
        rep = _lib.BatchReportC()
        if device:
            self.ctx.set_stream(torch.cuda.current_stream(x.device).cuda_stream)
        try:
            st = _lib.load().cfd_batch_linear_system_solve(self.h, C.byref(opt), bp, xp, res, C.byref(rep))
        finally:
            if device:
                self.ctx.set_stream(None)
        if st != _lib.CFD_OK:
            raise SolveError(f"batched linear-system solve failed: {_lib.STATUS_NAMES.get(st, st)}: "
                             f"{_lib.load().cfd_last_error().decode()}")
        arr = np.ctypeslib.as_array(res)[:self.num_systems]
        return xx, LinearSystemReport(rep.num_systems, rep.converged_systems, rep.total_iterations,
                                      rep.max_iterations, rep.max_rel_residual, rep.device_ms,
                                      arr["method"].astype(np.int32), arr["path"].astype(np.int32),
                                      arr["termination"].astype(np.int32), arr["iterations"].astype(np.int32),
                                      arr["residual"].astype(np.float64),
                                      {"direct": rep.direct_ms, "krylov": rep.krylov_ms,
                                       "fallback": rep.fallback_ms})

    def autotune(self, precision: Precision = Precision.FP64, sample_iterations: int = 64) -> dict:
        _lib.check(_lib.load().cfd_batch_autotune(self.h, int(precision), sample_iterations))
        return self.config(precision)

    def set_config(self, threads, systems_per_cta, precision: Precision = Precision.FP64) -> None:
        """Fix the Jacobi-PCG kernel's threads per system and systems per CTA
        for each of the 4 size buckets (in place of :meth:`autotune`)."""
        thr = np.ascontiguousarray(threads, dtype=np.int32)
        grp = np.ascontiguousarray(systems_per_cta, dtype=np.int32)
        if thr.shape != (4,) or grp.shape != (4,):
            raise ValueError("threads and systems_per_cta take one entry per bucket (4)")
        _lib.check(_lib.load().cfd_batch_set_config(self.h, int(precision), _p(thr), _p(grp)))

    def config(self, precision: Precision = Precision.FP64) -> dict:
        rows = np.zeros(4, np.int32)
        thr = np.zeros(4, np.int32)
        sysn = np.zeros(4, np.int32)
        grp = np.zeros(4, np.int32)
        _lib.check(_lib.load().cfd_batch_config(self.h, int(precision), _p(rows), _p(thr), _p(sysn)))
        _lib.check(_lib.load().cfd_batch_groups(self.h, int(precision), _p(grp)))
        return {"bucket_rows": rows.tolist(), "threads": thr.tolist(), "systems_per_cta": grp.tolist(),
                "systems": sysn.tolist()}

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            try:
                _lib.load().cfd_batch_destroy(h)
            except Exception:
                pass
            self.h = None


__all__ = ["NetworkBatch", "BatchReport", "LinearSystemReport", "LS_CG", "LS_BICGSTAB", "LS_DETECT", "LS_PATHS",
           "Termination", "PackedNetworks", "pack_networks", "network_assemble_host"]
