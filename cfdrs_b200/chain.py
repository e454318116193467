"""Tiered solve for saddle-point systems: ``LinearSolverChain``
(``crates/cfd-math/src/linear_solver/chain.rs``) over the tiers this package
provides.

The reference tries solvers in order and returns the first that converges
(``krylov::converged_or_none``); a tier whose setup fails, or whose solve ends
in an error or without converging, falls through to the next. Tiers built on
factorizations outside this package are skipped and recorded as such in
:attr:`LinearSolverChain.trace`:

* ``solve`` (``chain.rs:160-322``): direct LU [skipped], GMRES + component
  blocks (x reset to 0 after it), GMRES + SIMPLE (x reset to 0 after it), GMRES + AMG
  (``AMGConfig()``; x not reset, as in the reference), GMRES + block diagonal,
  GMRES unpreconditioned (from 0), GMRES + ILU [skipped], BiCGSTAB
  unpreconditioned (from 0; its failure fails the chain).
* ``solve_with_guess`` (``chain.rs:323-635``): direct LU [skipped], GMRES + SOR
  [skipped], GMRES + AMG (the hierarchy kept in a :class:`LinearSolverState`
  and recomputed for new values while the pattern is unchanged), GMRES +
  SIMPLE, GMRES + component blocks, GMRES + block diagonal, GMRES
  unpreconditioned only when no block-diagonal preconditioner could be built,
  GMRES + ILU [skipped], BiCGSTAB; every failed tier restarts the next from the
  initial guess.

GMRES restarts at ``min(krylov_restart, n)``. The solves run on the device
through :mod:`cfdrs_b200.krylov` with host arrays.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from . import krylov as K

SKIPPED = "skipped: not provided by this package"


class LinearSolverState:
    """``LinearSolverState``: the AMG hierarchy of the last warm solve and the
    pattern it was built for."""

    def __init__(self):
        self.amg = None
        self.pattern = None


class LinearSolverChain:
    """``LinearSolverChain::new(config)``; defaults direct_threshold = 2048,
    krylov_restart = 100 (``chain.rs:112-121``). The direct tier does not
    exist here, so the threshold only shows in the trace."""

    def __init__(self, config: K.IterativeSolverConfig):
        self.config = config
        self.direct_threshold = 2048
        self.krylov_restart = 100
        self.trace: list[tuple[str, str]] = []

    def with_direct_threshold(self, threshold: int) -> "LinearSolverChain":
        self.direct_threshold = int(threshold)
        return self

    def with_krylov_restart(self, restart: int) -> "LinearSolverChain":
        self.krylov_restart = int(restart)
        return self

    # Construction and solve hooks, looked up per call (tests replace them).
    def _simple(self, matrix, nv):
        from .saddle import SimplePreconditioner
        return SimplePreconditioner(matrix, nv)

    def _component_block(self, matrix, nv):
        from .saddle import ComponentBlockPreconditioner
        return ComponentBlockPreconditioner(matrix, nv)

    def _block_diagonal(self, matrix, nv):
        from .saddle import BlockDiagonalPreconditioner
        return BlockDiagonalPreconditioner(matrix, nv)

    def _amg(self, matrix):
        from .multigrid import AMGConfig, AlgebraicMultigrid
        return AlgebraicMultigrid(matrix, AMGConfig())

    def _gmres(self, matrix, rhs, pre, x, restart):
        if pre is None:
            return K.gmres(matrix, rhs, x, self.config, restart=restart)
        return K.gmres_preconditioned(matrix, rhs, pre, x, self.config, restart=restart)

    def _bicgstab(self, matrix, rhs, x):
        return K.bicgstab(matrix, rhs, x, self.config)

    def _attempt(self, name, run) -> bool:
        """One tier: True when it converged; setup and solve errors count as
        not converged, as ``converged_or_none`` treats an ``Err``."""
        try:
            rep = run()
        except (K.SolveError, _lib.CfdError) as e:
            self.trace.append((name, f"failed: {e}"))
            return False
        ok = K.converged_or_none(f"LinearSolverChain: {name}", rep) is not None
        self.trace.append((name, f"converged in {rep.iterations} iterations" if ok
                           else f"{rep.termination.name} after {rep.iterations} iterations"))
        return ok

    def _setup(self, name, make):
        try:
            return make()
        except (K.SolveError, _lib.CfdError) as e:
            self.trace.append((name, f"setup failed: {e}"))
            return None

    def solve(self, matrix, rhs, n_velocity_dof: int) -> np.ndarray:
        """``LinearSolverChain::solve`` (``chain.rs:160-322``)."""
        self.trace = []
        b = np.ascontiguousarray(rhs, dtype=np.float64)
        n = b.shape[0]
        restart = min(self.krylov_restart, max(n, 1))
        x = np.zeros(n)
        if n < self.direct_threshold:
            self.trace.append(("direct LU", SKIPPED))
        pre = self._setup("GMRES+ComponentBlock", lambda: self._component_block(matrix, n_velocity_dof))
        if pre is not None:
            if self._attempt("GMRES+ComponentBlock", lambda: self._gmres(matrix, b, pre, x, restart)):
                return x
            x[:] = 0.0
        pre = self._setup("GMRES+SIMPLE", lambda: self._simple(matrix, n_velocity_dof))
        if pre is not None:
            if self._attempt("GMRES+SIMPLE", lambda: self._gmres(matrix, b, pre, x, restart)):
                return x
            x[:] = 0.0
        pre = self._setup("GMRES+AMG", lambda: self._amg(matrix))
        if pre is not None and self._attempt("GMRES+AMG", lambda: self._gmres(matrix, b, pre, x, restart)):
            return x
        pre = self._setup("GMRES+BlockDiag", lambda: self._block_diagonal(matrix, n_velocity_dof))
        if pre is not None and self._attempt("GMRES+BlockDiag", lambda: self._gmres(matrix, b, pre, x, restart)):
            return x
        x[:] = 0.0
        if self._attempt("GMRES", lambda: self._gmres(matrix, b, None, x, restart)):
            return x
        x[:] = 0.0
        self.trace.append(("GMRES+ILU", SKIPPED))
        if self._attempt("BiCGSTAB", lambda: self._bicgstab(matrix, b, x)):
            return x
        raise K.SolveError("LinearSolverChain: all solver tiers failed")

    def solve_with_guess(self, matrix, rhs, n_velocity_dof: int, initial_guess=None,
                         state: LinearSolverState | None = None) -> np.ndarray:
        """``LinearSolverChain::solve_with_guess[_state]`` (``chain.rs:323-635``)."""
        self.trace = []
        state = state or LinearSolverState()
        b = np.ascontiguousarray(rhs, dtype=np.float64)
        n = b.shape[0]
        restart = min(self.krylov_restart, max(n, 1))
        guess = None if initial_guess is None else np.array(initial_guess, dtype=np.float64)
        x = np.zeros(n) if guess is None else guess.copy()

        def reset():
            x[:] = 0.0 if guess is None else guess

        if n < self.direct_threshold:
            self.trace.append(("direct LU", SKIPPED))
        self.trace.append(("GMRES+SOR", SKIPPED))
        pattern = (np.asarray(matrix.row_ptr).tobytes(), np.asarray(matrix.col).tobytes())

        def amg():
            if state.amg is not None and state.pattern == pattern:
                try:
                    state.amg.recompute(matrix)
                    return state.amg
                except (K.SolveError, _lib.CfdError):
                    pass  # rebuild, as the reference does when the cached hierarchy fails
            state.amg, state.pattern = None, None
            h = self._amg(matrix)
            state.amg, state.pattern = h, pattern
            return h
        pre = self._setup("GMRES+AMG", amg)
        if pre is not None:
            if self._attempt("GMRES+AMG", lambda: self._gmres(matrix, b, pre, x, restart)):
                return x
            reset()
        pre = self._setup("GMRES+SIMPLE", lambda: self._simple(matrix, n_velocity_dof))
        if pre is not None:
            if self._attempt("GMRES+SIMPLE", lambda: self._gmres(matrix, b, pre, x, restart)):
                return x
            reset()
        pre = self._setup("GMRES+ComponentBlock", lambda: self._component_block(matrix, n_velocity_dof))
        if pre is not None:
            if self._attempt("GMRES+ComponentBlock", lambda: self._gmres(matrix, b, pre, x, restart)):
                return x
            reset()
        pre = self._setup("GMRES+BlockDiag", lambda: self._block_diagonal(matrix, n_velocity_dof))
        if pre is not None:
            if self._attempt("GMRES+BlockDiag", lambda: self._gmres(matrix, b, pre, x, restart)):
                return x
            reset()
        else:
            if self._attempt("GMRES", lambda: self._gmres(matrix, b, None, x, restart)):
                return x
            reset()
        reset()
        self.trace.append(("GMRES+ILU", SKIPPED))
        if self._attempt("BiCGSTAB", lambda: self._bicgstab(matrix, b, x)):
            return x
        raise K.SolveError("LinearSolverChain: all solver tiers failed")


__all__ = ["LinearSolverChain", "LinearSolverState"]
