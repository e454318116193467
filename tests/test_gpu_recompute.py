"""Device Galerkin recompute (AlgebraicMultigrid::recompute, amg.rs:179-214):
with the transfer operators fixed, new fine values re-form every coarse
operator as (R_l A_l) P_l and the dense coarsest inverse, all on the device
(setup forms the coarsest inverse with the same device Gauss-Jordan).

The products are summed in the order of the reference-side Gustavson product
(terms of one output entry in the order of the left operand's row), the
inverse is Gauss-Jordan with partial pivoting step for step, so the device
results are compared bit for bit: against the oracle's SpGEMM chain on the
hierarchy's own R and P, and against a fresh setup where the hierarchy does
not depend on the values."""
import numpy as np
import pytest
import scipy.sparse as sp

from cfdrs_b200.sparse import CsrMatrix

pytestmark = pytest.mark.gpu


def from_scipy(m):
    m = sp.csr_matrix(m)
    m.sort_indices()
    return CsrMatrix(m.indptr.astype(np.int64), m.indices.astype(np.int64), m.data.astype(np.float64), m.shape)


def pressure_cfg(min_coarse):
    import cfdrs_b200 as cf
    cfg = cf.AMGConfig.pressure_poisson()
    cfg.min_coarse_size = min_coarse
    return cfg


def levels(amg):
    return [(amg.level(l, 0).row_ptr.copy(), amg.level(l, 0).col.copy(), amg.level(l, 0).val.copy())
            for l in range(amg.num_levels)]


@pytest.mark.parametrize("coarse", ["dense", "sweeps"])
def test_recompute_same_values_reproduces_setup(cuda, coarse):
    """Recompute with the setup's own values rebuilds the setup's hierarchy bit
    for bit (coarse operators, diagonals, coarsest inverse): the V-cycle output
    does not change in a single bit."""
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    A = P.poisson_3d_variable(16, 4.0, 1.0, seed=1)[0]
    cfg = pressure_cfg(100)
    if coarse == "sweeps":
        cfg.coarse_solve = cf.CoarseSolve.SWEEPS
    amg = cf.AlgebraicMultigrid(A, cfg)
    assert amg.num_levels >= 3
    before = levels(amg)
    r = np.random.default_rng(0).uniform(-1, 1, A.nrows)
    z0 = amg.apply_to(r)
    amg.recompute(A)
    after = levels(amg)
    for (rp0, c0, v0), (rp1, c1, v1) in zip(before, after):
        np.testing.assert_array_equal(rp0, rp1)
        np.testing.assert_array_equal(c0, c1)
        np.testing.assert_array_equal(v0, v1)
    np.testing.assert_array_equal(amg.apply_to(r), z0)


def test_recompute_matches_oracle_galerkin_chain(cuda, oracle):
    """New values: every level equals the oracle's (R_l A_l) P_l on the
    hierarchy's R_l, P_l, bit for bit, and the recomputed V-cycle is a working
    preconditioner for the new operator."""
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    A1 = P.poisson_3d_variable(16, 4.0, 1.0, seed=1)[0]
    A2, b2, _ = P.poisson_3d_variable(16, 3.0, 1.5, seed=7)
    assert np.array_equal(A1.col, A2.col) and not np.array_equal(A1.val, A2.val)
    amg = cf.AlgebraicMultigrid(A1, pressure_cfg(100))
    amg.recompute(A2)
    nl = amg.num_levels
    assert nl >= 3
    cur = oracle.Csr.from_matrix(A2)
    np.testing.assert_array_equal(amg.level(0, 0).val, A2.val)
    for l in range(nl - 1):
        R = oracle.Csr.from_matrix(amg.level(l, 2))
        Pm = oracle.Csr.from_matrix(amg.level(l, 1))
        cur = oracle.spgemm(oracle.spgemm(R, cur), Pm)
        rp, ci, v, shape = cur.arrays()
        dev = amg.level(l + 1, 0)
        np.testing.assert_array_equal(dev.row_ptr, rp)
        np.testing.assert_array_equal(dev.col, ci)
        np.testing.assert_array_equal(dev.val, v), f"level {l + 1}"
    x = np.zeros(A2.nrows)
    rep = cf.cg_preconditioned(A2, b2, amg, x, cf.IterativeSolverConfig(0.0, 1e-10, 200))
    assert rep.termination == cf.Termination.CONVERGED
    assert np.linalg.norm(A2.to_scipy() @ x - b2) <= 1e-9 * np.linalg.norm(b2)


def test_recompute_dense_inverse_bitwise(cuda):
    """One-level hierarchy (the V-cycle is the dense coarse solve): the inverse
    a recompute forms for the new values equals the one a fresh setup forms,
    bit for bit, and solves the new operator. Random nonsymmetric values force
    row exchanges at most pivots."""
    import cfdrs_b200 as cf
    n = 300
    rng = np.random.default_rng(11)
    pat = sp.random(n, n, density=0.04, random_state=5, format="csr") + sp.eye(n, format="csr")
    pat.data[:] = 1.0
    pat = sp.csr_matrix(pat)
    pat.sort_indices()

    def with_vals(seed):
        m = pat.copy()
        m.data = np.random.default_rng(seed).uniform(-1, 1, m.nnz)
        return from_scipy(m)

    A1, A2 = with_vals(1), with_vals(2)
    cfg = cf.AMGConfig(max_levels=1, coarse_solve=cf.CoarseSolve.DENSE)
    amg = cf.AlgebraicMultigrid(A1, cfg)
    assert amg.num_levels == 1
    amg.recompute(A2)
    fresh = cf.AlgebraicMultigrid(A2, cfg)
    r = rng.uniform(-1, 1, n)
    z = amg.apply_to(r)
    np.testing.assert_array_equal(z, fresh.apply_to(r))
    np.testing.assert_allclose(A2.to_scipy() @ z, r, atol=1e-8 * np.linalg.norm(r) * np.linalg.cond(
        A2.to_scipy().toarray()))


def test_recompute_singular_coarse_operator_fails(cuda):
    """A zero row keeps the pattern but makes the operator singular: the device
    elimination meets a zero pivot and the call fails with a status, as the
    host inverse does at setup."""
    import cfdrs_b200 as cf
    from cfdrs_b200._lib import CfdError
    from helpers import tridiag
    A1 = tridiag(64, -1.0, 3.0, -1.0)
    cfg = cf.AMGConfig(max_levels=1, coarse_solve=cf.CoarseSolve.DENSE)
    amg = cf.AlgebraicMultigrid(A1, cfg)
    v = A1.val.copy()
    v[A1.row_ptr[10]:A1.row_ptr[11]] = 0.0
    with pytest.raises(CfdError, match="singular"):
        amg.recompute(A1.with_values(v))
    with pytest.raises(CfdError, match="singular"):
        cf.AlgebraicMultigrid(A1.with_values(v), cfg)
    amg.recompute(A1)  # recovers with nonsingular values
    r = np.ones(64)
    np.testing.assert_allclose(A1.to_scipy() @ amg.apply_to(r), r, atol=1e-12)


def test_recompute_then_fp32_refinement(cuda):
    """FP32 copies of the level operators follow the recompute: FP32 inner CG
    inside FP64 refinement on the recomputed hierarchy meets the FP64 solution."""
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    A1 = P.poisson_3d_variable(20, 4.0, 1.0, seed=1)[0]
    A2, b2, _ = P.poisson_3d_variable(20, 5.0, 1.5, seed=3)
    amg = cf.AlgebraicMultigrid(A1, pressure_cfg(200))
    x = np.zeros(A1.nrows)
    cf.cg_preconditioned(A1, b2, amg, x, cf.IterativeSolverConfig(0.0, 1e-10, 300),
                         precision=cf.Precision.FP32_REFINE)  # creates the FP32 copies
    amg.recompute(A2)
    conf = cf.IterativeSolverConfig(0.0, 1e-10, 300)
    x64, x32 = np.zeros(A2.nrows), np.zeros(A2.nrows)
    r64 = cf.cg_preconditioned(A2, b2, amg, x64, conf)
    r32 = cf.cg_preconditioned(A2, b2, amg, x32, conf, precision=cf.Precision.FP32_REFINE)
    assert r64.termination == cf.Termination.CONVERGED and r32.termination == cf.Termination.CONVERGED
    assert np.linalg.norm(x32 - x64) <= 1e-8 * np.linalg.norm(x64)


def test_recompute_large_coarsest_inverse(cuda):
    """A 3843-row coarsest operator: more rows than the cooperative inverse
    has warps (148 SMs x 16), so warps take several rows per pivot step. A
    recompute with the setup's values reproduces the setup's inverse: the
    V-cycle output is unchanged bit for bit."""
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    A = P.poisson_3d_variable(36, 4.0, 1.0, seed=2)[0]
    amg = cf.AlgebraicMultigrid(A, pressure_cfg(4096))
    assert amg.statistics().level_sizes[-1] > 148 * 16
    r = np.random.default_rng(3).uniform(-1, 1, A.nrows)
    z0 = amg.apply_to(r)
    amg.recompute(A)
    np.testing.assert_array_equal(amg.apply_to(r), z0)


def test_recompute_leaves_other_matrices_alone(cuda):
    """A recompute reads the given matrix's values and changes no other
    matrix: after recomputing for A2, a solve with A1 still solves A1 (here
    with the hierarchy of A2 as its preconditioner)."""
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    A1, b1, _ = P.poisson_3d_variable(16, 4.0, 1.0, seed=1)
    A2 = P.poisson_3d_variable(16, 3.0, 1.5, seed=7)[0]
    amg = cf.AlgebraicMultigrid(A1, pressure_cfg(100))
    amg.recompute(A2)
    np.testing.assert_array_equal(amg.level(0, 0).val, A2.val)
    x = np.zeros(A1.nrows)
    rep = cf.cg_preconditioned(A1, b1, amg, x, cf.IterativeSolverConfig(0.0, 1e-10, 1000))
    assert rep.termination == cf.Termination.CONVERGED
    assert np.linalg.norm(A1.to_scipy() @ x - b1) <= 1e-9 * np.linalg.norm(b1)
