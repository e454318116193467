"""AMG preconditioner surface of cfd-math, backed by the device V-cycle.

Mirrors ``AMGConfig`` (``crates/cfd-math/src/linear_solver/preconditioners/
multigrid/mod.rs:219-259``), ``AlgebraicMultigrid::{new, recompute, apply_to}``
(``multigrid/amg.rs:133-214, 507-557``) and ``AMGStatistics``
(``multigrid/mod.rs:366-395``). The hierarchy is built on the host once
(coarsening, interpolation, Galerkin products) and lives on the device.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .device import Context, DeviceCsr, device_matrix
from .sparse import CsrMatrix


class CoarseningStrategy(enum.IntEnum):
    RUGE_STUEBEN = 0
    AGGREGATION = 1
    PMIS = 2


class InterpolationStrategy(enum.IntEnum):
    CLASSICAL = 0           # the reference formula, interpolation.rs:38-188
    DIRECT = 1              # piecewise constant, interpolation.rs:191-217
    MODIFIED_CLASSICAL = 2  # sign-restricted, lumps F-neighbours without a common C-point


class SmootherType(enum.IntEnum):
    JACOBI = 0


class CoarseOrder(enum.IntEnum):
    SELECTION = 0  # coarse index = selection order (the reference)
    ASCENDING = 1  # coarse points numbered by ascending fine index (local P/R gathers)


class CoarseSolve(enum.IntEnum):
    SWEEPS = 0  # smoother sweeps at the coarsest level (amg.rs:499-501)
    DENSE = 1   # exact FP64 solve with the dense inverse


@dataclass
class AMGConfig:
    """``AMGConfig`` with the device smoother (damped Jacobi)."""
    max_levels: int = 10
    min_coarse_size: int = 50
    coarsening_strategy: CoarseningStrategy = CoarseningStrategy.RUGE_STUEBEN
    interpolation_strategy: InterpolationStrategy = InterpolationStrategy.CLASSICAL
    smoother_type: SmootherType = SmootherType.JACOBI
    pre_smooth_iterations: int = 2
    post_smooth_iterations: int = 2
    relaxation_factor: float = 1.0
    strength_threshold: float = 0.25
    coarse_solve: CoarseSolve = CoarseSolve.SWEEPS
    coarse_sweeps: int = 10
    aggregate_size: int = 8
    seed: int = 0
    coarse_order: CoarseOrder = CoarseOrder.SELECTION
    # create_classical_interpolation's max_interpolation_points (interpolation.rs:42),
    # ignored by the reference: 0 keeps every weight; k > 0 keeps the k largest per
    # row of P, rescaled to the row sum.
    max_interpolation_points: int = 0

    @classmethod
    def pressure_poisson(cls) -> "AMGConfig":
        """V(1,1), damped Jacobi w = 2/3, coarsening to <= 4096 unknowns, exact
        FP64 coarsest solve, Ruge-Stueben coarsening with modified classical
        interpolation and ascending coarse numbering: the configuration of the
        3-D Poisson workloads."""
        return cls(max_levels=16, min_coarse_size=4096, pre_smooth_iterations=1, post_smooth_iterations=1,
                   relaxation_factor=2.0 / 3.0, coarse_solve=CoarseSolve.DENSE,
                   interpolation_strategy=InterpolationStrategy.MODIFIED_CLASSICAL,
                   coarse_order=CoarseOrder.ASCENDING)

    def to_c(self) -> _lib.AmgConfigC:
        return _lib.AmgConfigC(self.max_levels, int(self.coarsening_strategy), self.min_coarse_size,
                               int(self.interpolation_strategy), int(self.smoother_type),
                               self.pre_smooth_iterations, self.post_smooth_iterations, self.relaxation_factor,
                               self.strength_threshold, int(self.coarse_solve), self.coarse_sweeps,
                               self.aggregate_size, self.seed, int(self.coarse_order),
                               int(self.max_interpolation_points))


@dataclass
class AMGStatistics:
    num_levels: int
    level_sizes: list = field(default_factory=list)
    level_nnz: list = field(default_factory=list)
    operator_complexity: float = 1.0
    grid_complexity: float = 1.0
    setup_time: float = 0.0


class AlgebraicMultigrid:
    """``AlgebraicMultigrid::new(matrix, config)``; the device hierarchy handle."""

    def __init__(self, matrix, config: AMGConfig | None = None, ctx: Context | None = None):
        self.config = config or AMGConfig()
        self.matrix = device_matrix(matrix, ctx)
        self.ctx = self.matrix.ctx
        h = C.c_void_p()
        cfg = self.config.to_c()
        _lib.check(_lib.load().cfd_amg_setup(self.matrix.h, C.byref(cfg), C.byref(h)))
        self.h = h

    new = classmethod(lambda cls, matrix, config=None: cls(matrix, config))

    def recompute(self, matrix) -> None:
        """``AlgebraicMultigrid::recompute`` (amg.rs:179-214): re-form the
        Galerkin operators for the values of ``matrix`` (the setup's sparsity
        pattern), P and R kept. ``matrix`` is a host matrix (its device copy is
        made once, as for a solve) or a DeviceCsr on this hierarchy's context;
        the values of no other matrix change."""
        dm = device_matrix(matrix, self.ctx)
        _lib.check(_lib.load().cfd_amg_recompute(self.h, dm.h))

    def apply_to(self, r, z=None):
        """z = M^-1 r (one V-cycle from zero). Host numpy in/out, or CUDA torch tensors."""
        import torch
        if isinstance(r, torch.Tensor):
            out = torch.empty_like(r) if z is None else z
            _lib.check(_lib.load().cfd_amg_apply(self.h, C.c_void_p(r.data_ptr()), C.c_void_p(out.data_ptr())))
            return out
        rr = torch.as_tensor(np.ascontiguousarray(r, dtype=np.float64), device=f"cuda:{self.ctx.device}")
        zz = torch.empty_like(rr)
        torch.cuda.synchronize(self.ctx.device)
        _lib.check(_lib.load().cfd_amg_apply(self.h, C.c_void_p(rr.data_ptr()), C.c_void_p(zz.data_ptr())))
        res = zz.cpu().numpy()
        if z is not None:
            z[...] = res
            return z
        return res

    def set_path(self, path: str, fp32: bool) -> None:
        """SpMV pipeline of every level operator in one precision ("auto",
        "timed", "split", "record", "x_staged", "sliced", "diagonal"); an
        operator not eligible for the pipeline keeps "auto"; see DeviceCsr.set_path."""
        from .device import DeviceCsr
        _lib.check(_lib.load().cfd_amg_set_path(self.h, 1 if fp32 else 0, DeviceCsr.PATHS[path]))

    def statistics(self) -> AMGStatistics:
        return _statistics(self.h)

    def level(self, level: int, which: int = 0) -> CsrMatrix:
        """Host copy of level ``level``'s A (0), P (1) or R (2)."""
        return _level(self.h, level, which)

    @property
    def num_levels(self) -> int:
        return self.statistics().num_levels

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            try:
                _lib.load().cfd_amg_destroy(h)
            except Exception:
                pass
            self.h = None


def _statistics(h) -> AMGStatistics:
    s = _lib.AmgStatsC()
    _lib.check(_lib.load().cfd_amg_stats(h, C.byref(s)))
    n = s.num_levels
    return AMGStatistics(n, list(s.level_rows[:min(n, 16)]), list(s.level_nnz[:min(n, 16)]),
                         s.operator_complexity, s.grid_complexity, s.setup_seconds)


def _level(h, level: int, which: int) -> CsrMatrix:
    L = _lib.load()
    nr, nc, nnz = C.c_int64(), C.c_int64(), C.c_int64()
    _lib.check(L.cfd_amg_level(h, level, which, C.byref(nr), C.byref(nc), C.byref(nnz), None, None, None))
    rp = np.empty(nr.value + 1, np.int64)
    col = np.empty(nnz.value, np.int64)
    val = np.empty(nnz.value, np.float64)
    _lib.check(L.cfd_amg_level(h, level, which, None, None, None, rp.ctypes.data_as(C.c_void_p),
                               col.ctypes.data_as(C.c_void_p), val.ctypes.data_as(C.c_void_p)))
    return CsrMatrix(rp, col, val, (nr.value, nc.value))


class HostHierarchy:
    """The AMG hierarchy of ``AlgebraicMultigrid::new`` built on the host only
    (``cfd_amg_setup_host``): the same levels as :class:`AlgebraicMultigrid`
    without a device, for inspecting or serialising a hierarchy and for checking
    the setup where no GPU is present. It cannot precondition a solve."""

    def __init__(self, matrix, config: AMGConfig | None = None):
        m = matrix if isinstance(matrix, CsrMatrix) else CsrMatrix.from_scipy(matrix)
        if m.nrows != m.ncols:
            raise _lib.CfdError(1, "AMG needs a square matrix")
        self.config = config or AMGConfig()
        rp = np.ascontiguousarray(m.row_ptr, dtype=np.int64)
        col = np.ascontiguousarray(m.col, dtype=np.int64)
        val = np.ascontiguousarray(m.val, dtype=np.float64)
        h = C.c_void_p()
        cfg = self.config.to_c()
        _lib.check(_lib.load().cfd_amg_setup_host(m.nrows, rp.ctypes.data_as(C.c_void_p),
                                                  col.ctypes.data_as(C.c_void_p), val.ctypes.data_as(C.c_void_p),
                                                  C.byref(cfg), C.byref(h)))
        self.h = h

    def statistics(self) -> AMGStatistics:
        return _statistics(self.h)

    @property
    def num_levels(self) -> int:
        return self.statistics().num_levels

    def level(self, level: int, which: int = 0) -> CsrMatrix:
        """Level ``level``'s A (0), P (1) or R (2)."""
        return _level(self.h, level, which)

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            try:
                _lib.load().cfd_amg_destroy(h)
            except Exception:
                pass
            self.h = None


class JacobiPreconditioner:
    """``DiagJacobi`` / leto ``JacobiPreconditioner``: z = r / diag(A), identity
    where |a_ii| <= f64::EPSILON (``crates/cfd-1d/src/solver/core/linear_system.rs:270-332``)."""

    def __init__(self, matrix=None):
        self.matrix = matrix


class IdentityPreconditioner:
    """athena ``Identity`` (``krylov.rs:359``)."""
