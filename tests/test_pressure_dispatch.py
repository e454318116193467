"""The 2-D pressure-correction dispatch (correction.rs:40-168) on the CPU
with stub solvers: the AMG size limit, the cache keyed on the matrix values,
the retry without AMG after a breakdown, the kept iterate of a stalled solve,
and the solver choice (default GMRES(30))."""
import numpy as np
import pytest

from cfdrs_b200 import _lib
from cfdrs_b200 import krylov as K
from cfdrs_b200.pressure import AMG_SETUP_MATRIX_SIZE_LIMIT, PressureCorrectionDispatch, PressureLinearSolver
from cfdrs_b200.sparse import CsrMatrix

T = K.Termination


class Amg:
    def __init__(self):
        self.recomputed = []

    def recompute(self, matrix):
        self.recomputed.append(matrix.val.copy())


class Stub(PressureCorrectionDispatch):
    def __init__(self, outcomes, amg_fails=False, **kw):
        super().__init__(**kw)
        self.outcomes = list(outcomes)
        self.amg_fails = amg_fails
        self.built = 0
        self.calls = []

    def _new_amg(self, matrix):
        self.built += 1
        if self.amg_fails:
            raise _lib.CfdError(1, "setup refused")
        return Amg()

    def _solve(self, matrix, rhs, pre, solution):
        self.calls.append((pre is not None, np.array(solution, copy=True)))
        solution[...] = 7.0
        return K.SolveReport(self.outcomes.pop(0), 3, 1.0, 0.1, 0.01)


def matrix(n, scale=1.0):
    return CsrMatrix(np.arange(n + 1), np.arange(n), np.full(n, scale), (n, n))


def test_default_solver_is_gmres_30():
    d = PressureCorrectionDispatch()
    assert d.solver_type == PressureLinearSolver.gmres(30) and d.solver_type.restart_dim == 30


def test_amg_built_once_and_recomputed_only_for_new_values():
    d = Stub([T.CONVERGED] * 3)
    x = np.zeros(8)
    d.dispatch_solve(matrix(8), np.ones(8), x)
    d.dispatch_solve(matrix(8), np.ones(8), x)          # same values: nothing to redo
    d.dispatch_solve(matrix(8, 2.0), np.ones(8), x)     # new values: recompute, no new setup
    assert d.built == 1 and len(d.amg.recomputed) == 1 and d.amg.recomputed[0][0] == 2.0
    assert all(pre for pre, _ in d.calls)


def test_size_limit_skips_amg():
    n = AMG_SETUP_MATRIX_SIZE_LIMIT
    d = Stub([T.CONVERGED])
    d.dispatch_solve(matrix(n), np.ones(n), np.zeros(n))
    assert d.built == 0 and d.calls[0][0] is False
    d = Stub([T.CONVERGED])
    d.dispatch_solve(matrix(n - 1), np.ones(n - 1), np.zeros(n - 1))
    assert d.built == 1 and d.calls[0][0] is True


def test_failed_setup_solves_without_amg_and_retries_setup_next_time():
    d = Stub([T.CONVERGED, T.CONVERGED], amg_fails=True)
    d.dispatch_solve(matrix(8), np.ones(8), np.zeros(8))
    d.dispatch_solve(matrix(8), np.ones(8), np.zeros(8))
    assert d.built == 2 and not any(pre for pre, _ in d.calls)


def test_breakdown_with_amg_retries_without_it_from_zero():
    d = Stub([T.BREAKDOWN, T.CONVERGED])
    x = np.full(8, 3.0)
    out = d.dispatch_solve(matrix(8), np.ones(8), x)
    assert [pre for pre, _ in d.calls] == [True, False]
    assert np.all(d.calls[0][1] == 3.0) and np.all(d.calls[1][1] == 0.0)
    assert out.converged()


def test_stalled_or_broken_down_keeps_the_last_iterate():
    for outcomes, kind in (([T.MAX_ITERATIONS], K.SolveOutcome.STALLED),
                           ([T.BREAKDOWN, T.NON_POSITIVE_CURVATURE], K.SolveOutcome.BROKEN_DOWN)):
        d = Stub(outcomes)
        x = np.zeros(8)
        out = d.dispatch_solve(matrix(8), np.ones(8), x)
        assert out.kind == kind and np.all(x == 7.0)


def test_breakdown_without_amg_is_not_retried():
    d = Stub([T.BREAKDOWN], amg_fails=True)
    out = d.dispatch_solve(matrix(8), np.ones(8), np.zeros(8))
    assert len(d.calls) == 1 and out.kind == K.SolveOutcome.BROKEN_DOWN


def test_csr_values_are_read_only_and_set_values_bumps_the_version():
    from helpers import tridiag
    A = tridiag(5)
    with pytest.raises(ValueError):
        A.val[0] = 7.0
    v0 = A.version
    A.set_values(2.0 * np.asarray(A.val))
    assert A.version == v0 + 1 and np.array_equal(A.val, 2.0 * tridiag(5).val)
    with pytest.raises(ValueError):
        A.set_values(np.ones(3))
