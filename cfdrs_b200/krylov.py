"""Krylov entry points mirroring ``cfd_math::linear_solver::krylov``
(``crates/cfd-math/src/linear_solver/krylov.rs``), solved on the device.

* ``cg_preconditioned`` / ``bicgstab_preconditioned`` / ``cg`` / ``bicgstab``
  (``krylov.rs:253-360``) take ``(matrix, rhs, [preconditioner,] solution,
  config)``; ``solution`` carries the initial guess in and the result out.
* Dimension / configuration / backend failures raise :class:`SolveError`
  (the reference's ``Err``); numerical end states come back in the
  :class:`SolveReport` (``Ok(SolveReport)``), classified by :func:`interpret`
  (``krylov.rs:375-401``) into :class:`SolveOutcome`.
* ``precision=Precision.FP32_REFINE`` runs FP32 inner Krylov/AMG solves inside
  FP64 iterative refinement.

Convergence: threshold = max(tolerance, relative_tolerance * ||r0||), the
absolute-or-relative test of ``crates/cfd-core/src/compute/solver/convergence.rs:26-30``.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass

import numpy as np

from . import _lib
from .device import device_matrix
from .multigrid import AlgebraicMultigrid, IdentityPreconditioner, JacobiPreconditioner


class SolveError(RuntimeError):
    """``SolveError`` / ``cfd_core::error::Error::Solver``."""


class Termination(enum.IntEnum):
    CONVERGED = 0
    INITIAL_RESIDUAL = 1
    MAX_ITERATIONS = 2
    BREAKDOWN = 3
    NON_POSITIVE_CURVATURE = 4


class Precision(enum.IntEnum):
    FP64 = 0
    FP32_REFINE = 1


@dataclass
class IterativeSolverConfig:
    """``IterativeSolverConfig``: absolute tolerance, relative tolerance (vs ||r0||)
    and iteration budget."""
    tolerance: float = 1e-6
    relative_tolerance: float = 0.0
    max_iterations: int = 1000

    @classmethod
    def new(cls, tolerance: float) -> "IterativeSolverConfig":
        return cls(tolerance=tolerance)

    def with_max_iterations(self, n: int) -> "IterativeSolverConfig":
        self.max_iterations = n
        return self

    def with_relative_tolerance(self, rtol: float) -> "IterativeSolverConfig":
        self.relative_tolerance = rtol
        return self

    def to_c(self) -> _lib.SolverConfigC:
        return _lib.SolverConfigC(self.tolerance, self.relative_tolerance, self.max_iterations)


@dataclass
class SolveReport:
    termination: Termination
    iterations: int
    initial_residual_norm: float
    final_residual_norm: float
    threshold: float
    outer_iterations: int = 0
    device_ms: float = 0.0


class SolveOutcome:
    """``SolveOutcome::{Converged, Stalled, BrokenDown}`` (``krylov.rs:403-428``)."""

    CONVERGED, STALLED, BROKEN_DOWN = "Converged", "Stalled", "BrokenDown"

    def __init__(self, kind: str, report: SolveReport):
        self.kind = kind
        self.report = report

    def converged(self) -> bool:
        return self.kind == self.CONVERGED

    def __repr__(self):
        return f"SolveOutcome.{self.kind}({self.report})"


def interpret(context: str, report: SolveReport) -> SolveOutcome:
    """``krylov::interpret``: Converged / InitialResidual -> Converged,
    MaxIterations -> Stalled, Breakdown / NonPositiveCurvature -> BrokenDown."""
    t = report.termination
    if t in (Termination.CONVERGED, Termination.INITIAL_RESIDUAL):
        return SolveOutcome(SolveOutcome.CONVERGED, report)
    if t == Termination.MAX_ITERATIONS:
        return SolveOutcome(SolveOutcome.STALLED, report)
    if t in (Termination.BREAKDOWN, Termination.NON_POSITIVE_CURVATURE):
        return SolveOutcome(SolveOutcome.BROKEN_DOWN, report)
    raise SolveError(f"{context}: linear solve terminated as {t!r}")


def converged_or_none(context: str, report: SolveReport) -> SolveReport | None:
    """``krylov::converged_or_none`` (``krylov.rs:501-523``)."""
    out = interpret(context, report)
    return report if out.converged() else None


_SOLVER_CG, _SOLVER_BICGSTAB, _SOLVER_GMRES = 0, 1, 2
_PRE_NONE, _PRE_JACOBI, _PRE_AMG, _PRE_SIMPLE, _PRE_BLOCK_DIAGONAL, _PRE_COMPONENT_BLOCK = 0, 1, 2, 3, 4, 5
_SADDLE_PRE = {"SimplePreconditioner": _PRE_SIMPLE, "BlockDiagonalPreconditioner": _PRE_BLOCK_DIAGONAL,
               "ComponentBlockPreconditioner": _PRE_COMPONENT_BLOCK}


def _solve(solver: int, matrix, rhs, preconditioner, solution, config: IterativeSolverConfig,
           precision: Precision = Precision.FP64, inner_tolerance: float = 1e-4, check_every: int = 0,
           max_outer: int = 20, restart: int = 30) -> SolveReport:
    import torch
    L = _lib.load()
    amg_h = None
    if preconditioner is None or isinstance(preconditioner, IdentityPreconditioner):
        pre = _PRE_NONE
    elif isinstance(preconditioner, JacobiPreconditioner):
        pre = _PRE_JACOBI
    elif isinstance(preconditioner, AlgebraicMultigrid):
        pre = _PRE_AMG
        amg_h = preconditioner.h
    elif type(preconditioner).__name__ in _SADDLE_PRE:
        pre = _SADDLE_PRE[type(preconditioner).__name__]
        if preconditioner.matrix is not matrix:
            raise SolveError("the saddle-point preconditioner was set up on another matrix object")
    else:
        raise SolveError(f"unsupported preconditioner {type(preconditioner).__name__}")
    dm = device_matrix(matrix, preconditioner.ctx if pre in (_PRE_AMG, _PRE_SIMPLE, _PRE_BLOCK_DIAGONAL, _PRE_COMPONENT_BLOCK)
                       else None)
    n = dm.shape[0]
    if restart < 1:
        raise SolveError(f"GMRES restart must be positive, got {restart}")
    opt = _lib.SolveOptionsC(solver, pre, int(precision), 0, inner_tolerance, max_outer, check_every, restart)
    rep = _lib.SolveReportC()
    cfg = config.to_c()
    if isinstance(solution, torch.Tensor):
        if not (isinstance(rhs, torch.Tensor) and rhs.is_cuda and solution.is_cuda):
            raise SolveError("device solves need CUDA tensors for both rhs and solution")
        if rhs.dtype != torch.float64 or solution.dtype != torch.float64:
            raise SolveError("device solves take float64 tensors")
        if rhs.numel() != n or solution.numel() != n:
            raise SolveError(f"dimension mismatch: matrix {n}, rhs {rhs.numel()}, solution {solution.numel()}")
        opt.memory = 1
        dm.ctx.set_stream(torch.cuda.current_stream(solution.device).cuda_stream)
        try:
            status = L.cfd_solve(dm.h, C.byref(opt), amg_h, C.c_void_p(rhs.contiguous().data_ptr()),
                                 C.c_void_p(solution.data_ptr()), C.byref(cfg), C.byref(rep))
        finally:
            dm.ctx.set_stream(None)
    else:
        b = np.ascontiguousarray(rhs, dtype=np.float64)
        if b.shape[0] != n or solution.shape[0] != n:
            raise SolveError(f"dimension mismatch: matrix {n}, rhs {b.shape[0]}, solution {solution.shape[0]}")
        x = np.ascontiguousarray(solution, dtype=np.float64)
        status = L.cfd_solve(dm.h, C.byref(opt), amg_h, b.ctypes.data_as(C.c_void_p),
                             x.ctypes.data_as(C.c_void_p), C.byref(cfg), C.byref(rep))
        if x is not solution:
            solution[...] = x
    if status != _lib.CFD_OK:
        msg = L.cfd_last_error().decode()
        raise SolveError(f"linear solve failed: {_lib.STATUS_NAMES.get(status, status)}: {msg}")
    return SolveReport(Termination(rep.termination), rep.iterations, rep.initial_residual, rep.final_residual,
                       rep.threshold, rep.outer_iterations, rep.device_ms)


def cg_preconditioned(matrix, rhs, preconditioner, solution, config, **kw) -> SolveReport:
    """``krylov::cg_preconditioned`` (``krylov.rs:318-343``)."""
    return _solve(_SOLVER_CG, matrix, rhs, preconditioner, solution, config, **kw)


def cg(matrix, rhs, solution, config, **kw) -> SolveReport:
    """``krylov::cg`` (``krylov.rs:350-360``)."""
    return _solve(_SOLVER_CG, matrix, rhs, None, solution, config, **kw)


def bicgstab_preconditioned(matrix, rhs, preconditioner, solution, config, **kw) -> SolveReport:
    """``krylov::bicgstab_preconditioned`` (``krylov.rs:253-278``)."""
    return _solve(_SOLVER_BICGSTAB, matrix, rhs, preconditioner, solution, config, **kw)


def bicgstab(matrix, rhs, solution, config, **kw) -> SolveReport:
    """``krylov::bicgstab`` (``krylov.rs:285-308``)."""
    return _solve(_SOLVER_BICGSTAB, matrix, rhs, None, solution, config, **kw)


def gmres_preconditioned(matrix, rhs, preconditioner, solution, config, restart: int = 30, **kw) -> SolveReport:
    """``krylov::gmres_preconditioned`` (``krylov.rs:150-170``): restarted GMRES,
    right preconditioned, the restart rounded up the ladder 8, 16, ..., 256."""
    return _solve(_SOLVER_GMRES, matrix, rhs, preconditioner, solution, config, restart=restart, **kw)


def gmres(matrix, rhs, solution, config, restart: int = 30, **kw) -> SolveReport:
    """``krylov::gmres`` (``krylov.rs:228-246``)."""
    return _solve(_SOLVER_GMRES, matrix, rhs, None, solution, config, restart=restart, **kw)


def gmres_width(requested: int) -> int:
    """``RestartWidth::covering`` (``krylov.rs:96-120``): the smallest of 8, 16,
    32, 64, 128, 256 covering the request, saturating at 256."""
    w = 8
    while w < 256 and w < requested:
        w *= 2
    return w


class SolverKind:
    """``SolverKind`` (``krylov.rs:533-612``): ConjugateGradient, BiCgStab or
    Gmres { restart } (``SolverKind.gmres(restart)``)."""
    CONJUGATE_GRADIENT: "SolverKind"
    BICGSTAB: "SolverKind"

    def __init__(self, kind: str, restart: int | None = None):
        self.kind = kind
        self.restart = restart

    @classmethod
    def gmres(cls, restart: int) -> "SolverKind":
        return cls("GMRES", restart)

    def name_(self) -> str:
        return self.kind

    def __eq__(self, other) -> bool:
        return isinstance(other, SolverKind) and (self.kind, self.restart) == (other.kind, other.restart)

    def __hash__(self) -> int:
        return hash((self.kind, self.restart))

    def __repr__(self) -> str:
        return f"SolverKind.{self.kind}" + (f"{{restart: {self.restart}}}" if self.kind == "GMRES" else "")

    def solve(self, matrix, rhs, solution, config, **kw) -> SolveReport:
        if self.kind == "GMRES":
            return gmres(matrix, rhs, solution, config, self.restart, **kw)
        f = cg if self.kind == "ConjugateGradient" else bicgstab
        return f(matrix, rhs, solution, config, **kw)

    def solve_preconditioned(self, matrix, rhs, preconditioner, solution, config, **kw) -> SolveReport:
        if self.kind == "GMRES":
            return gmres_preconditioned(matrix, rhs, preconditioner, solution, config, self.restart, **kw)
        f = cg_preconditioned if self.kind == "ConjugateGradient" else bicgstab_preconditioned
        return f(matrix, rhs, preconditioner, solution, config, **kw)


SolverKind.CONJUGATE_GRADIENT = SolverKind("ConjugateGradient")
SolverKind.BICGSTAB = SolverKind("BiCGSTAB")
