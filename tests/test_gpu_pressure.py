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


def test_dispatch_sees_values_changed_in_place(cuda):
    """A SIMPLE loop reuses one matrix and changes its values between calls:
    the recompute and the solve must read the new values, whether they came in
    through CsrMatrix.set_values or were written into the caller's own array."""
    import scipy.sparse.linalg as spla
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.pressure import PressureCorrectionDispatch
    from cfdrs_b200.sparse import CsrMatrix
    A0, b = P.poisson_2d_dirichlet(48)
    own = np.array(A0.val)  # the caller's value array, held by reference
    A = CsrMatrix(A0.row_ptr, A0.col, own, A0.shape)
    d = PressureCorrectionDispatch(config=cf.IterativeSolverConfig(0.0, 1e-10, 2000))
    x = np.zeros(A.shape[0])
    assert d.dispatch_solve(A, b, x).converged()
    rng = np.random.default_rng(3)
    # the direct write first: set_values gives the matrix its own copy, after
    # which the caller's array is no longer the matrix's
    for scale_rows, direct in ((rng.uniform(0.5, 2.0, A.shape[0]), True), (rng.uniform(0.5, 2.0, A.shape[0]), False)):
        S = A0.to_scipy()
        Dh = np.sqrt(scale_rows)
        new = (S.multiply(Dh[:, None]).multiply(Dh[None, :])).tocsr()  # stays SPD, same pattern
        new.sort_indices()
        if direct:
            assert np.shares_memory(A.val, own)
            own[:] = new.data
        else:
            A.set_values(new.data)
        x = np.zeros(A.shape[0])
        assert d.dispatch_solve(A, b, x).converged()
        x_ref = spla.spsolve(new.tocsc(), b)
        assert np.linalg.norm(x - x_ref) <= 1e-8 * np.linalg.norm(x_ref)
    assert d.recomputes == 2


def test_solve_after_set_values_uses_the_new_values(cuda):
    import scipy.sparse.linalg as spla
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    A, b = P.poisson_2d_dirichlet(40)
    x = np.zeros(A.shape[0])
    cfg = cf.IterativeSolverConfig(0.0, 1e-12, 4000)
    assert cf.cg_preconditioned(A, b, cf.JacobiPreconditioner(A), x, cfg).termination == cf.Termination.CONVERGED
    A.set_values(3.0 * np.asarray(A.val))
    x = np.zeros(A.shape[0])
    assert cf.cg_preconditioned(A, b, cf.JacobiPreconditioner(A), x, cfg).termination == cf.Termination.CONVERGED
    x_ref = spla.spsolve(A.to_scipy().tocsc(), b)
    assert np.linalg.norm(x - x_ref) <= 1e-9 * np.linalg.norm(x_ref)
