"""Device GMRES(m) (krylov::gmres_preconditioned, krylov.rs:150-246) against the
reference's GMRES tests and against the CPU oracle's restatement of the same
recurrence (restart ladder, CGS2 Arnoldi, Givens rotations, true residual at
every restart)."""
import numpy as np
import pytest

from helpers import csr_from_lists, grid_laplacian, manufactured, tridiag
from test_oracle_golden import gmres_golden_cases

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_gmres_reference_cases(cuda, golden):
    import cfdrs_b200 as cf
    g = golden["gmres_diagonal_2"]
    A = csr_from_lists(g["row_ptr"], g["col"], g["val"])
    for _ in range(2):  # the reference reuses one workspace for two solves
        x = np.zeros(2)
        rep = cf.gmres(A, np.array(g["b"]), x, cf.IterativeSolverConfig(g["tolerance"], 0.0, g["max_iterations"]),
                       restart=g["restart"])
        assert rep.final_residual_norm <= rep.threshold
        np.testing.assert_allclose(x, g["x"], atol=g["tol"])
    for name, M, b, g in gmres_golden_cases(golden):
        x = np.zeros_like(b)
        rep = cf.gmres(M, b, x, cf.IterativeSolverConfig(g["tolerance"], 0.0, g["max_iterations"]),
                       restart=g["restart"])
        assert rep.termination == cf.Termination.CONVERGED, name
        assert np.linalg.norm(M.to_scipy() @ x - b) < g["residual_below"], name


def test_amg_gmres_reference(cuda, golden):
    """amg_integration_test.rs:125-142 on the device V-cycle (damped Jacobi)."""
    import cfdrs_b200 as cf
    g = golden["amg_gmres_2d_16"]
    A = grid_laplacian(g["n"])
    xs = manufactured(A.nrows)
    amg = cf.AlgebraicMultigrid(A, cf.AMGConfig(relaxation_factor=2 / 3))
    x = np.zeros(A.nrows)
    rep = cf.SolverKind.gmres(g["restart"]).solve_preconditioned(
        A, A.matvec(xs), amg, x, cf.IterativeSolverConfig(g["tolerance"], 0.0, g["max_iterations"]))
    assert rep.termination == cf.Termination.CONVERGED
    assert np.max(np.abs(x - xs)) < g["max_abs_error"]


@pytest.mark.parametrize("pre", ["none", "jacobi"])
def test_gmres_matches_oracle_nonsymmetric(cuda, oracle, pre):
    """Nonsymmetric tridiagonal system, GMRES(8) with many restarts: the device
    and the oracle take the same number of steps (to one, at the threshold) and
    reach the same solution."""
    import cfdrs_b200 as cf
    n = 3000
    A = tridiag(n, lo=-1.3, d=3.0, hi=-0.7)
    b = np.random.default_rng(3).uniform(-1, 1, n)
    opre = {"none": oracle.PRE_NONE, "jacobi": oracle.PRE_JACOBI}[pre]
    xo, ro = oracle.gmres(oracle.Csr.from_matrix(A), b, restart=8, precond=opre, rtol=1e-10, max_it=2000)
    assert ro.termination == "Converged"
    x = np.zeros(n)
    cfg = cf.IterativeSolverConfig(0.0, 1e-10, 2000)
    if pre == "none":
        rep = cf.gmres(A, b, x, cfg, restart=8)
    else:
        rep = cf.gmres_preconditioned(A, b, cf.JacobiPreconditioner(A), x, cfg, restart=8)
    assert rep.termination == cf.Termination.CONVERGED
    assert abs(rep.iterations - ro.iterations) <= 1
    assert rel(x, xo) < 1e-8
    assert rep.final_residual_norm <= rep.threshold


@pytest.mark.parametrize("precision", ["fp64", "fp32_refine"])
def test_amg_gmres_3d(cuda, oracle, precision):
    """3-D variable-coefficient Poisson with the pressure AMG: device GMRES(30)
    FP64 against the oracle's GMRES(30) on the same hierarchy definition (same
    step count to one, same solution), and FP32 inner GMRES inside FP64
    refinement to 1e-8 of the FP64 solution."""
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    A, b, _ = P.poisson_3d_variable(24, 8.0, 1.0, seed=5)
    cfgm = cf.AMGConfig.pressure_poisson()
    cfgm.min_coarse_size = 200
    amg = cf.AlgebraicMultigrid(A, cfgm)
    oamg = oracle.Amg(oracle.Csr.from_matrix(A), oracle.AmgConfig(
        max_levels=16, min_coarse_size=200, smoother=oracle.SMOOTH_JACOBI, pre_smooth=1, post_smooth=1,
        relaxation=2 / 3, coarse_solve=oracle.COARSE_DENSE, interpolation=2, coarse_order=1))
    xo, ro = oracle.gmres(oracle.Csr.from_matrix(A), b, restart=30, precond=oracle.PRE_AMG, amg=oamg,
                          rtol=1e-10, max_it=500)
    assert ro.termination == "Converged"
    x64 = np.zeros(A.nrows)
    rep64 = cf.gmres_preconditioned(A, b, amg, x64, cf.IterativeSolverConfig(0.0, 1e-10, 500))
    assert rep64.termination == cf.Termination.CONVERGED
    assert abs(rep64.iterations - ro.iterations) <= 1
    assert rel(x64, xo) < 1e-9
    if precision == "fp32_refine":
        x = np.zeros(A.nrows)
        rep = cf.gmres_preconditioned(A, b, amg, x, cf.IterativeSolverConfig(0.0, 1e-10, 500),
                                      precision=cf.Precision.FP32_REFINE)
        assert rep.termination == cf.Termination.CONVERGED and rep.outer_iterations >= 1
        assert rel(x, x64) < 1e-8


def test_gmres_termination_and_ladder(cuda):
    import cfdrs_b200 as cf
    n = 500
    A = tridiag(n, lo=-1.3, d=3.0, hi=-0.7)
    b = np.random.default_rng(4).uniform(-1, 1, n)
    x = np.zeros(n)
    rep = cf.gmres(A, b, x, cf.IterativeSolverConfig(0.0, 1e-14, 5), restart=8)
    assert rep.termination == cf.Termination.MAX_ITERATIONS and rep.iterations == 5
    x = np.zeros(n)
    rep = cf.gmres(A, np.zeros(n), x, cf.IterativeSolverConfig(0.0, 1e-8, 50))
    assert rep.termination == cf.Termination.INITIAL_RESIDUAL and rep.iterations == 0
    # restart 3 and 8 both run GMRES(8): identical results
    x3, x8 = np.zeros(n), np.zeros(n)
    r3 = cf.gmres(A, b, x3, cf.IterativeSolverConfig(0.0, 1e-10, 1000), restart=3)
    r8 = cf.gmres(A, b, x8, cf.IterativeSolverConfig(0.0, 1e-10, 1000), restart=8)
    assert cf.gmres_width(3) == 8 and r3.iterations == r8.iterations and np.array_equal(x3, x8)
    with pytest.raises(cf.SolveError):
        cf.gmres(A, b, np.zeros(n), cf.IterativeSolverConfig(0.0, 1e-10, 10), restart=0)


def test_gmres_device_tensors(cuda):
    """Device pointers (torch tensors on the current stream) give the host-buffer result."""
    import cfdrs_b200 as cf
    n = 2000
    A = tridiag(n, lo=-1.3, d=3.0, hi=-0.7)
    b = np.random.default_rng(6).uniform(-1, 1, n)
    xh = np.zeros(n)
    cfg = cf.IterativeSolverConfig(0.0, 1e-10, 1000)
    cf.gmres(A, b, xh, cfg, restart=16)
    bd = cuda.as_tensor(b, device="cuda")
    xd = cuda.zeros_like(bd)
    cf.gmres(A, bd, xd, cfg, restart=16)
    cuda.cuda.synchronize()
    np.testing.assert_array_equal(xd.cpu().numpy(), xh)
