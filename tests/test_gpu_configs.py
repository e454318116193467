"""The plain FP64 path against the oracle on the 3-D configurations at the
coarsening limit they name (min_coarse_size 4096): the drop-in contract of
``krylov::cg_preconditioned`` (crates/cfd-math/src/linear_solver/krylov.rs:318-343)
with the AMG preconditioner of amg.rs:423-503 is a solution equal to the CPU
solve's to a relative difference of 1e-10 at an equal residual tolerance.

The oracle builds its own hierarchy from the same matrix (no export from the
device); both solve from x = 0 to a 1e-8 relative residual. The full 256^3
systems are compared by ``bench.py --workload c2|c3`` (its ``oracle_parity``
block); these tests run 128^3 (2.1 M unknowns), which the oracle sets up and
solves in seconds.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _oracle_amg(O, Ao):
    return O.Amg(Ao, O.AmgConfig(max_levels=16, min_coarse_size=4096, smoother=O.SMOOTH_JACOBI, pre_smooth=1,
                                 post_smooth=1, relaxation=2 / 3, coarse_solve=O.COARSE_DENSE, interpolation=2,
                                 coarse_order=1))


def _check(cuda, oracle, A, b):
    import cfdrs_b200 as cf
    amg = cf.AlgebraicMultigrid(A, cf.AMGConfig.pressure_poisson())
    Ao = oracle.Csr.from_matrix(A)
    oamg = _oracle_amg(oracle, Ao)
    st = amg.statistics()
    assert st.num_levels == oamg.num_levels
    for l in range(st.num_levels):
        r, _, z = oamg.level(l).info()
        assert (st.level_sizes[l], st.level_nnz[l]) == (r, z)
    xo, ro = oracle.pcg(Ao, b, precond=oracle.PRE_AMG, amg=oamg, rtol=1e-8, max_it=500)
    x = np.zeros_like(b)
    rep = cf.cg_preconditioned(A, b, amg, x, cf.IterativeSolverConfig(0.0, 1e-8, 500))
    assert rep.termination == cf.Termination.CONVERGED and ro.termination == "Converged"
    assert rep.iterations == ro.iterations
    assert _rel(x, xo) <= 1e-10
    assert np.linalg.norm(b - A.matvec(x)) <= 1.0000001e-8 * np.linalg.norm(b)
    return amg, x, rep


def test_c2_constant_coefficient_128_matches_the_oracle(cuda, oracle):
    """C2's system (7-point FV, Dirichlet x = 0 and 1, Neumann elsewhere, k = 1,
    b ~ U[-1, 1]) at 128^3."""
    from cfdrs_b200 import problems as P
    A, b = P.poisson_3d_fv(128, seed=0)
    _check(cuda, oracle, A, b)


def test_c3_variable_coefficient_128_fp64_matches_the_oracle_and_fp32_refinement_is_within_1e8(cuda, oracle):
    """C3's system (k = exp(GRF), l = 8 cells, sigma = 1) at 128^3: the FP64
    solve equals the oracle's; FP32 inner AMG-PCG inside FP64 refinement to
    1e-10 is within 1e-8 of the oracle's FP64 solve driven to 1e-12."""
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    A, b, _ = P.poisson_3d_variable(128, 8.0, 1.0, seed=0)
    amg, _, _ = _check(cuda, oracle, A, b)
    Ao = oracle.Csr.from_matrix(A)
    xo, ro = oracle.pcg(Ao, b, precond=oracle.PRE_AMG, amg=_oracle_amg(oracle, Ao), rtol=1e-12, max_it=500)
    x = np.zeros_like(b)
    rep = cf.cg_preconditioned(A, b, amg, x, cf.IterativeSolverConfig(0.0, 1e-10, 500),
                               precision=cf.Precision.FP32_REFINE)
    assert rep.termination == cf.Termination.CONVERGED
    assert _rel(x, xo) <= 1e-8
