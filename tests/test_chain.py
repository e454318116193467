"""LinearSolverChain's orchestration on the CPU (chain.rs): tier order, which
tiers restart from zero or the guess and which continue from the previous
iterate, setup failures and solve errors falling through, the final error,
and the warm AMG state. The solvers and preconditioner constructors are
replaced by stubs; the device solves of the tiers are covered by the GPU
tests of each preconditioner."""
import numpy as np
import pytest

from cfdrs_b200 import _lib
from cfdrs_b200 import krylov as K
from cfdrs_b200.chain import SKIPPED, LinearSolverChain, LinearSolverState
from cfdrs_b200.sparse import CsrMatrix

CONV, STALL, BREAK = K.Termination.CONVERGED, K.Termination.MAX_ITERATIONS, K.Termination.BREAKDOWN


class Amg:
    def __init__(self):
        self.recomputed = 0

    def recompute(self, matrix):
        self.recomputed += 1


class StubChain(LinearSolverChain):
    """Each tier's solve writes a distinct marker into x and records the x it
    started from; outcomes[name] is a termination or an exception."""
    MARK = {"SIMPLE": 1.0, "AMG": 2.0, "BlockDiag": 3.0, None: 4.0, "BiCGSTAB": 5.0, "ComponentBlock": 6.0}

    def __init__(self, outcomes, failing_setups=()):
        super().__init__(K.IterativeSolverConfig(0.0, 1e-8, 100))
        self.outcomes = outcomes
        self.failing_setups = set(failing_setups)
        self.calls = []
        self.amg_built = 0

    def _make(self, name, obj):
        if name in self.failing_setups:
            raise _lib.CfdError(1, f"{name} setup refused")
        return obj

    def _simple(self, matrix, nv):
        return self._make("SIMPLE", "SIMPLE")

    def _block_diagonal(self, matrix, nv):
        return self._make("BlockDiag", "BlockDiag")

    def _component_block(self, matrix, nv):
        return self._make("ComponentBlock", "ComponentBlock")

    def _amg(self, matrix):
        self.amg_built += 1
        return self._make("AMG", Amg())

    def _run(self, name, x):
        self.calls.append((name, x.copy()))
        x[:] = self.MARK[name]
        out = self.outcomes.get(name, STALL)
        if isinstance(out, Exception):
            raise out
        return K.SolveReport(out, 7, 1.0, 0.5, 0.1)

    def _gmres(self, matrix, rhs, pre, x, restart):
        assert restart == min(self.krylov_restart, x.shape[0])
        return self._run("AMG" if isinstance(pre, Amg) else pre, x)

    def _bicgstab(self, matrix, rhs, x):
        return self._run("BiCGSTAB", x)


def matrix(n=6):
    return CsrMatrix(np.arange(n + 1), np.arange(n), np.ones(n), (n, n))


def names(chain):
    return [c[0] for c in chain.calls]


def test_cold_order_and_first_success():
    ch = StubChain({"AMG": CONV})
    x = ch.solve(matrix(), np.ones(6), 4)
    assert names(ch) == ["ComponentBlock", "SIMPLE", "AMG"] and np.all(x == 2.0)
    assert ch.trace[0] == ("direct LU", SKIPPED) and ch.trace[1][0] == "GMRES+ComponentBlock"
    assert ch.trace[-1][0] == "GMRES+AMG" and ch.trace[-1][1].startswith("converged")


def test_cold_resets_follow_the_reference():
    """From 0 after the component blocks and SIMPLE; the block diagonal
    continues from AMG's iterate; unpreconditioned GMRES and BiCGSTAB start
    from 0."""
    ch = StubChain({"BiCGSTAB": CONV})
    ch.solve(matrix(), np.ones(6), 4)
    assert names(ch) == ["ComponentBlock", "SIMPLE", "AMG", "BlockDiag", None, "BiCGSTAB"]
    starts = {n: x for n, x in ch.calls}
    assert np.all(starts["ComponentBlock"] == 0)
    assert np.all(starts["SIMPLE"] == 0) and np.all(starts["AMG"] == 0)
    assert np.all(starts["BlockDiag"] == 2.0)
    assert np.all(starts[None] == 0) and np.all(starts["BiCGSTAB"] == 0)
    assert ("GMRES+ILU", SKIPPED) in ch.trace


def test_cold_setup_failures_and_errors_fall_through():
    ch = StubChain({"SIMPLE": K.SolveError("boom"), "BlockDiag": BREAK, None: CONV},
                   failing_setups={"AMG", "ComponentBlock"})
    x = ch.solve(matrix(), np.ones(6), 4)
    assert names(ch) == ["SIMPLE", "BlockDiag", None] and np.all(x == 4.0)
    trace = dict(ch.trace)
    assert trace["GMRES+ComponentBlock"].startswith("setup failed")
    assert trace["GMRES+SIMPLE"].startswith("failed") and trace["GMRES+AMG"].startswith("setup failed")
    assert trace["GMRES+BlockDiag"].startswith("BREAKDOWN")


def test_cold_all_tiers_fail():
    ch = StubChain({})
    with pytest.raises(K.SolveError, match="all solver tiers failed"):
        ch.solve(matrix(), np.ones(6), 4)
    assert names(ch) == ["ComponentBlock", "SIMPLE", "AMG", "BlockDiag", None, "BiCGSTAB"]


def test_restart_is_capped_by_the_size():
    ch = StubChain({"SIMPLE": CONV}).with_krylov_restart(30)
    ch.solve(matrix(6), np.ones(6), 4)  # the stub asserts restart == min(30, 6)
    ch = StubChain({"SIMPLE": CONV}).with_krylov_restart(3)
    ch.solve(matrix(6), np.ones(6), 4)


def test_warm_order_resets_to_the_guess_and_skips_gmres():
    """AMG first, then SIMPLE, the component blocks and the block diagonal;
    each restarts from the guess; unpreconditioned GMRES only runs when no
    block diagonal could be built."""
    guess = np.full(6, 9.0)
    ch = StubChain({"BiCGSTAB": CONV})
    ch.solve_with_guess(matrix(), np.ones(6), 4, guess)
    assert names(ch) == ["AMG", "SIMPLE", "ComponentBlock", "BlockDiag", "BiCGSTAB"]
    assert all(np.all(x == 9.0) for _, x in ch.calls)
    assert ch.trace[1] == ("GMRES+SOR", SKIPPED)
    ch = StubChain({None: CONV}, failing_setups={"BlockDiag"})
    x = ch.solve_with_guess(matrix(), np.ones(6), 4, guess)
    assert names(ch) == ["AMG", "SIMPLE", "ComponentBlock", None] and np.all(x == 4.0)
    assert np.all(dict(ch.calls)[None] == 9.0)


def test_warm_state_keeps_the_hierarchy_for_the_same_pattern():
    state = LinearSolverState()
    ch = StubChain({"AMG": CONV})
    A = matrix()
    ch.solve_with_guess(A, np.ones(6), 4, None, state)
    first = state.amg
    ch.solve_with_guess(A.with_values(2.0 * A.val), np.ones(6), 4, None, state)
    assert ch.amg_built == 1 and state.amg is first and first.recomputed == 1
    B = CsrMatrix(np.array([0, 2, 3, 4, 5, 6, 7]), np.array([0, 1, 1, 2, 3, 4, 5]), np.ones(7), (6, 6))
    ch.solve_with_guess(B, np.ones(6), 4, None, state)
    assert ch.amg_built == 2 and state.amg is not first
