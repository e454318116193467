"""The 2-D pressure-correction caller of the solve path:
``PressureCorrectionSolver::dispatch_solve``
(``crates/cfd-2d/src/pressure_velocity/correction.rs:40-168``) with its solver
choice ``PressureLinearSolver`` (``pressure_velocity/config.rs:15-34``).

Per call: below ``AMG_SETUP_MATRIX_SIZE_LIMIT`` rows an AMG hierarchy
(``AMGConfig()``) is built once and afterwards recomputed (Galerkin operators
for the new values, on the device) only when the matrix values differ from
the ones it was last formed for; a failed first setup leaves the solve
unpreconditioned. The configured Krylov method runs with the hierarchy; a
breakdown with AMG is retried from zero without it. A stalled or broken-down
final solve keeps its last iterate (the reference logs and returns ``Ok``);
an unknown termination raises.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib
from . import krylov as K
from .device import refresh_device_values

AMG_SETUP_MATRIX_SIZE_LIMIT = 10_000


@dataclass(frozen=True)
class PressureLinearSolver:
    """``PressureLinearSolver``: ``conjugate_gradient``, ``bicgstab`` or
    ``gmres(restart_dim)``; the default is GMRES(30)."""
    kind: str = "gmres"
    restart_dim: int = 30

    @classmethod
    def conjugate_gradient(cls) -> "PressureLinearSolver":
        return cls("cg", 0)

    @classmethod
    def bicgstab(cls) -> "PressureLinearSolver":
        return cls("bicgstab", 0)

    @classmethod
    def gmres(cls, restart_dim: int = 30) -> "PressureLinearSolver":
        return cls("gmres", int(restart_dim))


class PressureCorrectionDispatch:
    """The solver part of ``PressureCorrectionSolver``: its solver choice, its
    linear-solver configuration (here by default an absolute tolerance of
    1e-10 and 1000 iterations; the reference takes it from the solver's
    configuration) and its AMG cache (``_amg_preconditioner``,
    ``_amg_matrix_values``)."""

    def __init__(self, solver_type: PressureLinearSolver | None = None,
                 config: K.IterativeSolverConfig | None = None):
        self.solver_type = solver_type or PressureLinearSolver()
        self.linear_solver_config = config or K.IterativeSolverConfig(1e-10, 0.0, 1000)
        self.amg = None
        self.amg_values = None
        self.solved_values = None
        self.recomputes = 0
        self.last_outcome: K.SolveOutcome | None = None

    # Hooks, looked up per call (tests replace them).
    def _new_amg(self, matrix):
        from .multigrid import AMGConfig, AlgebraicMultigrid
        return AlgebraicMultigrid(matrix, AMGConfig())

    def _solve(self, matrix, rhs, pre, solution) -> K.SolveReport:
        cfg, t = self.linear_solver_config, self.solver_type
        if t.kind == "cg":
            return K.cg_preconditioned(matrix, rhs, pre, solution, cfg) if pre else K.cg(matrix, rhs, solution, cfg)
        if t.kind == "bicgstab":
            return (K.bicgstab_preconditioned(matrix, rhs, pre, solution, cfg) if pre
                    else K.bicgstab(matrix, rhs, solution, cfg))
        if pre:
            return K.gmres_preconditioned(matrix, rhs, pre, solution, cfg, restart=t.restart_dim)
        return K.gmres(matrix, rhs, solution, cfg, restart=t.restart_dim)

    def dispatch_solve(self, matrix, rhs, solution) -> K.SolveOutcome:
        """Solves into ``solution`` (a host array or CUDA tensor) and returns
        the final outcome."""
        values = np.asarray(matrix.val)
        if self.solved_values is not None and not np.array_equal(self.solved_values, values):
            # values written into the matrix's array since the last call (also
            # directly, bypassing CsrMatrix.set_values): push them to the
            # device copy that the recompute and the solve read
            refresh_device_values(matrix)
        self.solved_values = values.copy()
        unchanged = (self.amg is not None and self.amg_values is not None
                     and np.array_equal(self.amg_values, values))
        allowed = matrix.shape[0] < AMG_SETUP_MATRIX_SIZE_LIMIT
        if allowed and not unchanged:
            if self.amg is None:
                try:
                    self.amg = self._new_amg(matrix)
                except (K.SolveError, _lib.CfdError, ValueError):
                    # the reference keeps going without AMG on any Err of
                    # AlgebraicMultigrid::new (`if let Ok(amg)`, correction.rs:63-80)
                    self.amg = None
            else:
                self.amg.recompute(matrix)  # an error here propagates, as the reference's `?` does
                self.recomputes += 1
            if self.amg is not None:
                self.amg_values = values.copy()
        pre = self.amg
        outcome = K.interpret("pressure correction", self._solve(matrix, rhs, pre, solution))
        if outcome.kind == K.SolveOutcome.BROKEN_DOWN and pre is not None:
            solution[...] = 0.0
            outcome = K.interpret("pressure correction", self._solve(matrix, rhs, None, solution))
        self.last_outcome = outcome
        return outcome


__all__ = ["AMG_SETUP_MATRIX_SIZE_LIMIT", "PressureCorrectionDispatch", "PressureLinearSolver"]
