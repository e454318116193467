"""The 2-D pressure-correction dispatch on the device: GMRES(30) + AMG on a
64 x 64 pressure Poisson system (below the AMG size limit), the hierarchy
kept for unchanged values and recomputed on the device for new ones, and no
AMG above the limit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_dispatch_with_cached_amg(cuda):
    import scipy.sparse.linalg as spla
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.pressure import PressureCorrectionDispatch
    A, b = P.poisson_2d_dirichlet(64)
    d = PressureCorrectionDispatch(config=cf.IterativeSolverConfig(0.0, 1e-10, 2000))
    x = np.zeros(A.shape[0])
    out = d.dispatch_solve(A, b, x)
    assert out.converged() and d.amg is not None
    x_ref = spla.spsolve(A.to_scipy().tocsc(), b)
    assert np.linalg.norm(x - x_ref) <= 1e-8 * np.linalg.norm(x_ref)
    amg = d.amg
    x[:] = 0.0
    d.dispatch_solve(A, b, x)
    assert d.amg is amg and d.recomputes == 0
    A2 = A.with_values(2.0 * A.val)
    x2 = np.zeros(A.shape[0])
    assert d.dispatch_solve(A2, b, x2).converged()
    assert d.amg is amg and d.recomputes == 1
    assert np.linalg.norm(2.0 * x2 - x_ref) <= 1e-8 * np.linalg.norm(x_ref)


def test_dispatch_above_the_limit_runs_without_amg(cuda):
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.krylov import SolveOutcome
    from cfdrs_b200.pressure import AMG_SETUP_MATRIX_SIZE_LIMIT, PressureCorrectionDispatch
    A, b = P.poisson_2d_dirichlet(101)
    assert A.shape[0] >= AMG_SETUP_MATRIX_SIZE_LIMIT
    d = PressureCorrectionDispatch(config=cf.IterativeSolverConfig(0.0, 1e-8, 300))
    x = np.zeros(A.shape[0])
    out = d.dispatch_solve(A, b, x)
    assert d.amg is None and out.kind in (SolveOutcome.CONVERGED, SolveOutcome.STALLED)
    assert np.linalg.norm(x) > 0  # a stalled solve keeps its last iterate
