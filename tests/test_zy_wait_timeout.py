"""Failure detection without a GPU fault: a bounded device wait (the mbarrier
wait every bulk-copy SpMV pipeline uses) runs out on a barrier nothing
completes, the host call reports CFD_ERR_TIMEOUT with the wait's message, and
the context stays usable (a solve on it afterwards converges)."""
import numpy as np
import pytest

from helpers import tridiag

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_context_stays_usable(cuda):
    import cfdrs_b200 as cf
    from cfdrs_b200 import _lib
    from cfdrs_b200.device import context
    ctx = context(0)
    L = _lib.load()
    assert L.cfd_selftest_wait_timeout(ctx.h, 1000) == 4  # CFD_ERR_TIMEOUT
    assert b"bounded wait ran out" in L.cfd_last_error()
    n = 1000
    A = tridiag(n)
    b = np.ones(n)
    x = np.zeros(n)
    rep = cf.cg(A, b, x, cf.IterativeSolverConfig(0.0, 1e-10, 5000))
    assert rep.termination == cf.Termination.CONVERGED
    assert np.linalg.norm(A.to_scipy() @ x - b) <= 1e-9 * np.linalg.norm(b)
    assert L.cfd_selftest_wait_timeout(ctx.h, 0) == 2  # CFD_ERR_CONFIG: no wait at all
