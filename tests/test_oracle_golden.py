"""Pins the CPU oracle against the reference's own known-answer tests
(tests/golden/reference_golden.json) and against scipy as an independent referee."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

from helpers import csr_from_lists, grid_laplacian, manufactured, tridiag


def test_smoother_golden_vectors(oracle, golden):
    g = golden["smoother_tridiagonal_5"]
    A = oracle.Csr.from_matrix(tridiag(5))
    x0, b = np.array(g["x0"]), np.array(g["b"])
    for kind, key in [(oracle.SMOOTH_JACOBI, "jacobi"), (oracle.SMOOTH_GS, "gauss_seidel"),
                      (oracle.SMOOTH_SGS, "symmetric_gauss_seidel"), (oracle.SMOOTH_GS, "sor_1")]:
        x = oracle.smooth(A, x0, b, kind, g["relaxation"], g["sweeps"])
        np.testing.assert_array_equal(x, np.array(g[key]), err_msg=key)


def test_strength_golden(oracle, golden):
    g = golden["strength_grid_4x4"]
    S = oracle.strength(oracle.Csr.from_matrix(grid_laplacian(4)), g["theta"])
    rp, ci, v, _ = S.arrays()
    assert rp[-1] == g["nnz"]
    assert list(ci[rp[0]:rp[1]]) == g["row0_cols"] and list(v[rp[0]:rp[1]]) == g["row0_vals"]
    assert list(ci[rp[5]:rp[6]]) == g["row5_cols"] and list(v[rp[5]:rp[6]]) == g["row5_vals"]


def test_spmv_golden(oracle, golden):
    g = golden["spmv_3x3"]
    A = oracle.Csr.from_matrix(csr_from_lists(g["row_ptr"], g["col"], g["val"]))
    np.testing.assert_allclose(A.spmv(np.array(g["x"])), g["y"], atol=g["tol"])


def test_coarsest_dense_golden(oracle, golden):
    g = golden["coarsest_solve_3x3"]
    A = oracle.Csr.from_matrix(csr_from_lists(g["row_ptr"], g["col"], g["val"]))
    np.testing.assert_allclose(oracle.dense_solve(A, np.array(g["b"])), g["x"], atol=g["tol"])


@pytest.mark.parametrize("solver", ["pcg", "bicgstab"])
def test_diagonal_solve_golden(oracle, golden, solver):
    g = golden["diagonal_solve_2"]
    A = oracle.Csr.from_matrix(csr_from_lists(g["row_ptr"], g["col"], g["val"]))
    fn = getattr(oracle, solver)
    for _ in range(2):  # reusable-workspace test runs the solve twice
        x, rep = fn(A, np.array(g["b"]), tol=g["tolerance"], rtol=0.0, max_it=g["max_iterations"])
        assert rep.final_residual <= rep.threshold
        np.testing.assert_allclose(x, g["x"], atol=g["tol"])


def test_amg_integration_bicgstab(oracle, golden):
    """amg_integration_test.rs:97-122 with AMGConfig::default (RS, classical, GS 2/2)."""
    g = golden["amg_poisson_2d_16"]
    n = g["n"]
    A = grid_laplacian(n)
    xs = manufactured(n * n)
    b = A.matvec(xs)
    Ao = oracle.Csr.from_matrix(A)
    amg = oracle.Amg(Ao, oracle.AmgConfig())
    x, rep = oracle.bicgstab(Ao, b, precond=oracle.PRE_AMG, amg=amg, tol=g["tolerance"], rtol=0.0,
                             max_it=g["max_iterations"])
    assert rep.termination == "Converged"
    assert np.max(np.abs(x - xs)) < g["max_abs_error"]
    x, rep = oracle.pcg(Ao, b, precond=oracle.PRE_AMG, amg=oracle.Amg(Ao, oracle.AmgConfig(
        smoother=oracle.SMOOTH_JACOBI, relaxation=2 / 3, pre_smooth=1, post_smooth=1)),
        tol=g["tolerance"], rtol=0.0, max_it=g["max_iterations"])
    assert rep.termination == "Converged" and np.max(np.abs(x - xs)) < g["max_abs_error"]


def test_amg_contraction(oracle, golden):
    """amg_integration_test.rs:212-268: stationary AMG iteration contracts in the A-norm."""
    g = golden["amg_poisson_2d_16"]
    for n in g["contraction_sizes"]:
        A = grid_laplacian(n)
        S = A.to_scipy()
        xs = manufactured(n * n)
        b = S @ xs
        Ao = oracle.Csr.from_matrix(A)
        amg = oracle.Amg(Ao, oracle.AmgConfig())
        x = np.zeros(n * n)
        en = lambda v: np.sqrt(max(v @ (S @ v), 0.0))  # noqa: E731
        prev, worst = en(xs - x), 0.0
        for _ in range(g["contraction_steps"]):
            x = x + amg.apply(b - S @ x)
            e = en(xs - x)
            worst = max(worst, e / prev)
            prev = e
            if e == 0:
                break
        assert worst < g["contraction_bound"]


def test_amg_single_level_and_depth_cap(oracle):
    """amg_integration_test.rs:170-209: tiny matrix -> one level, still nonzero z; max_levels=1 honoured."""
    A = oracle.Csr.from_matrix(grid_laplacian(4))
    amg = oracle.Amg(A, oracle.AmgConfig())
    assert amg.num_levels == 1
    assert np.any(amg.apply(manufactured(16)) != 0)
    deep = oracle.Amg(oracle.Csr.from_matrix(grid_laplacian(16)), oracle.AmgConfig(max_levels=1))
    assert deep.num_levels == 1


def test_ruge_stueben_tree_matches_reference_scan(oracle):
    """The O(log n) tournament pick equals the reference's first-maximum scan (algorithms.rs:64-74)."""
    from cfdrs_b200 import problems as P
    for A in [grid_laplacian(9), P.poisson_3d_fv(6)[0], P.poisson_3d_variable(8, 2.0, 1.0, seed=3)[0]]:
        Ao = oracle.Csr.from_matrix(A)
        cp_fast, f_fast = oracle.coarsen(Ao, oracle.RUGE_STUEBEN, 0.25, literal_scan=False)
        cp_lit, f_lit = oracle.coarsen(Ao, oracle.RUGE_STUEBEN, 0.25, literal_scan=True)
        np.testing.assert_array_equal(cp_fast, cp_lit)
        np.testing.assert_array_equal(f_fast, f_lit)


def test_pcg_against_scipy(oracle):
    from cfdrs_b200 import problems as P
    A, b = P.poisson_2d_dirichlet(32, seed=4)
    Ao = oracle.Csr.from_matrix(A)
    x, rep = oracle.pcg(Ao, b, precond=oracle.PRE_JACOBI, rtol=1e-12, max_it=2000)
    assert rep.termination == "Converged"
    xs = spla.spsolve(A.to_scipy().tocsc(), b)
    np.testing.assert_allclose(x, xs, rtol=1e-9, atol=1e-10)


def test_bicgstab_nonsymmetric_against_scipy(oracle):
    n = 200
    rng = np.random.default_rng(0)
    A = tridiag(n, lo=-1.3, d=3.0, hi=-0.7)
    b = rng.uniform(-1, 1, n)
    x, rep = oracle.bicgstab(oracle.Csr.from_matrix(A), b, precond=oracle.PRE_JACOBI, rtol=1e-12, max_it=500)
    assert rep.termination == "Converged"
    np.testing.assert_allclose(x, spla.spsolve(A.to_scipy().tocsc(), b), rtol=1e-9, atol=1e-10)


def test_termination_mapping(oracle):
    from cfdrs_b200 import problems as P
    A, b = P.poisson_2d_dirichlet(16, seed=1)
    Ao = oracle.Csr.from_matrix(A)
    _, rep = oracle.pcg(Ao, b, precond=oracle.PRE_JACOBI, rtol=1e-12, max_it=1)
    assert rep.termination == "MaxIterations" and rep.iterations == 1
    _, rep = oracle.pcg(Ao, np.zeros_like(b), precond=oracle.PRE_JACOBI, rtol=1e-8, max_it=10)
    assert rep.termination == "InitialResidual" and rep.iterations == 0
    neg = csr_from_lists([0, 1, 2], [0, 1], [-1.0, -2.0])
    _, rep = oracle.pcg(oracle.Csr.from_matrix(neg), np.array([1.0, 1.0]), precond=oracle.PRE_NONE, rtol=1e-8)
    assert rep.termination == "NonPositiveCurvature"


def test_jacobi_tiny_diagonal(oracle, golden):
    """linear_system.rs:339-349: |d| <= eps gives identity for that row."""
    g = golden["jacobi_tiny_diagonal"]
    A = oracle.Csr.from_matrix(csr_from_lists(g["row_ptr"], g["col"], g["val"]))
    b = np.array([3.0, 4.0])
    x, rep = oracle.pcg(A, b, precond=oracle.PRE_JACOBI, rtol=0.0, tol=1e-30, max_it=1)
    # one PCG step with z = inv_diag * r from x = 0: x = alpha * z
    z = np.array(g["inv_diag"]) * b
    alpha = (b @ z) / (z @ np.array([1e-18 * z[0], 2.0 * z[1]]))
    np.testing.assert_allclose(x, alpha * z, rtol=1e-12)


def test_kirchhoff_abc_golden(golden):
    from cfdrs_b200 import problems as P
    g = golden["kirchhoff_abc"]
    e = np.array(g["edges"])
    dirichlet = {int(k): v for k, v in g["dirichlet"].items()}
    A, b = P.kirchhoff_assemble(3, e[:, 0].astype(int), e[:, 1].astype(int), e[:, 2], dirichlet)
    D = A.to_scipy().toarray()
    assert abs(D[1, 1] - g["diag_b"]) < g["tol"] and abs(b[1] - g["rhs_b"]) < g["tol"]
    assert D[0, 0] == 1.0 and D[2, 2] == 1.0 and b[0] == 100.0 and b[2] == 0.0
    assert D[1, 0] == 0.0 and D[1, 2] == 0.0
    _, b5 = P.kirchhoff_assemble(3, e[:, 0].astype(int), e[:, 1].astype(int), e[:, 2], dirichlet, {1: 5.0})
    assert abs(b5[1] - g["rhs_b_with_neumann_5"]) < g["tol"]


def _oracle_network(oracle, edges, dirichlet, n, neumann=None):
    e = np.array(edges)
    fixed, value = np.zeros(n, np.int8), np.zeros(n)
    for k, v in dirichlet.items():
        fixed[int(k)], value[int(k)] = 1, v
    q = None
    if neumann:
        q = np.zeros(n)
        for k, v in neumann.items():
            q[k] = v
    A, b = oracle.network_assemble(n, e[:, 0], e[:, 1], e[:, 2], fixed, value, q)
    return A.to_scipy().toarray(), b


def test_oracle_network_assembly_golden(oracle, golden):
    """or_network_assemble on the reference's assembly tests
    (matrix_assembly.rs:270-450): identity rows for fixed nodes, Dirichlet
    columns eliminated into the RHS, the Neumann source, the free block."""
    g = golden["kirchhoff_abc"]
    D, b = _oracle_network(oracle, g["edges"], g["dirichlet"], 3)
    assert D[1, 1] == g["diag_b"] and b[1] == g["rhs_b"]
    assert D[0, 0] == 1.0 and D[2, 2] == 1.0 and b[0] == 100.0 and b[2] == 0.0
    assert D[1, 0] == 0.0 and D[1, 2] == 0.0 and D[0, 1] == 0.0 and D[2, 1] == 0.0
    _, b5 = _oracle_network(oracle, g["edges"], g["dirichlet"], 3, {1: 5.0})
    assert b5[1] == g["rhs_b_with_neumann_5"] and b5[0] == 100.0  # the fixed row keeps p
    g = golden["kirchhoff_active_block"]
    D, b = _oracle_network(oracle, g["edges"], g["dirichlet"], 4)
    assert np.array_equal(D, np.array(g["dense"])) and np.array_equal(b, np.array(g["rhs"]))


@pytest.mark.parametrize("bad,kind", [((1, 1, 1.0), "self-loop"), ((0, 2, np.nan), "non-finite"),
                                      ((0, 2, np.inf), "non-finite"), ((0, 2, 0.0), "non-positive"),
                                      ((0, 2, -1.0), "non-positive")])
def test_oracle_network_assembly_rejects(oracle, bad, kind):
    """matrix_assembly.rs:184-203: the first offending edge is reported."""
    with pytest.raises(ValueError, match=f"{kind}.*at edge 1"):
        _oracle_network(oracle, [(0, 1, 1.0), bad, (1, 2, 2.0)], {0: 1.0}, 3)


def test_oracle_network_assembly_parallel_edges_and_sources(oracle):
    """Parallel edges merge into one entry per (row, column), summed in edge
    order; a free node with several fixed neighbours sums g p in edge order;
    an edge between two fixed nodes contributes nothing; every node may carry
    a Neumann source, fixed rows ignore theirs."""
    edges = [(0, 1, 0.1), (1, 2, 0.2), (2, 1, 0.3), (1, 3, 0.7), (3, 4, 1.1), (4, 0, 1.3), (2, 4, 1.7),
             (1, 2, 0.9)]
    D, b = _oracle_network(oracle, edges, {0: 3.0, 4: -2.0}, 5, {1: 0.5, 2: -0.25, 4: 9.0})
    assert D[1, 2] == (-0.2 + -0.3) + -0.9 and D[2, 1] == D[1, 2]
    assert D[1, 1] == (((0.1 + 0.2) + 0.3) + 0.7) + 0.9
    assert D[2, 2] == ((0.2 + 0.3) + 1.7) + 0.9
    assert D[3, 3] == 0.7 + 1.1 and D[3, 4] == 0.0 and D[0, 0] == 1.0 and D[4, 4] == 1.0
    assert b[1] == 0.1 * 3.0 + 0.5 and b[2] == 1.7 * -2.0 + -0.25 and b[3] == 1.1 * -2.0
    assert b[0] == 3.0 and b[4] == -2.0


def test_oracle_network_assembly_matches_problem_assembly(oracle):
    """The oracle and problems.kirchhoff_assemble (scipy's COO merge) give the
    same pattern and, up to the order of the diagonal sums, the same values on
    the seeded C4-style networks."""
    from cfdrs_b200 import problems as P
    for net in P.network_batch_edges(12, seed=5, n_min=20, n_max=800):
        A, b = net.assemble()
        O, ob = oracle.network_assemble(net.n_nodes, net.edges_i, net.edges_j, net.conductance, net.fixed,
                                        net.fixed_value)
        rp, ci, v, _ = O.arrays()
        assert np.array_equal(rp, A.row_ptr) and np.array_equal(ci, A.col)
        np.testing.assert_allclose(v, A.val, rtol=4e-16 * 16, atol=0)
        assert np.array_equal(ob, b)


def test_equilibrated_pcg_networks(oracle):
    """Jacobi-PCG with the 1-D solver's equilibrated residual test reaches the
    direct solution on seeded networks (linear_system.rs:157-204)."""
    from cfdrs_b200 import problems as P
    for A, b in P.network_batch(6, seed=2, n_min=20, n_max=400):
        x, rep = oracle.pcg_equilibrated(oracle.Csr.from_matrix(A), b, rtol=1e-12)
        assert rep.termination == "Converged"
        xs = spla.spsolve(A.to_scipy().tocsc(), b)
        assert np.linalg.norm(x - xs) <= 1e-6 * np.linalg.norm(xs)


def test_cpu_adjoint_against_fd_and_assembly():
    """The CPU adjoint oracle: its assembly equals problems.darcy_2d and the
    torch assembly, and its hand-derived gradient matches central differences."""
    import adjoint_cpu as AC
    import torch
    from cfdrs_b200 import problems as P
    from cfdrs_b200.adjoint import darcy_2d_pattern, darcy_2d_torch, loss_column_index
    n = 20
    theta = P.gaussian_random_field((n, n), 3.0, 0.5, seed=3)
    A1, b1 = P.darcy_2d(theta)
    A2, b2 = AC.assemble(theta)
    assert abs(A1.to_scipy() - A2).max() <= 1e-14 and np.array_equal(b1, b2)
    _, mask = darcy_2d_pattern(n)
    vals, bt = darcy_2d_torch(torch.as_tensor(theta), torch.as_tensor(mask))
    assert np.array_equal(vals.numpy(), A1.val) and np.array_equal(bt.numpy(), b1)
    col = loss_column_index(n)
    _, g, _ = AC.loss_and_grad(theta, col)
    cells = [(1, 2), (5, col), (n - 1, n - 1), (7, 0), (10, 13)]
    fd = AC.central_fd(theta, col, cells)
    ga = np.array([g[j, i] for j, i in cells])
    assert np.abs(ga - fd).max() <= 1e-6 * np.abs(g).max()
    # the Woodbury route to the same differences (corner, wall and interior cells)
    fd_lr = AC.central_fd_lowrank(theta, col, cells)
    assert np.abs(fd_lr - fd).max() <= 1e-6 * np.abs(g).max()
    assert np.abs(ga - fd_lr).max() <= 1e-7 * np.abs(g).max()


def _entries_csr(n, entries):
    import scipy.sparse as sp
    from cfdrs_b200.sparse import CsrMatrix
    e = np.array(entries, dtype=float)
    return CsrMatrix.from_scipy(sp.csr_matrix((e[:, 2], (e[:, 0].astype(int), e[:, 1].astype(int))), shape=(n, n)))


def gmres_golden_cases(golden):
    """(name, matrix, b, restart, tolerance, max_iterations, residual bound) of
    the reference's GMRES tests (simple_gmres_tests.rs, core_solver_tests.rs)."""
    cases = []
    g = golden["gmres_basic_5"]
    cases.append(("basic_5", _entries_csr(g["n"], g["entries"]), np.array(g["b"]), g))
    g = golden["gmres_restart_8"]
    cases.append(("restart_8", tridiag(g["n"]), np.ones(g["n"]), g))
    g = golden["gmres_diag_precond_6"]
    cases.append(("diag_6", _entries_csr(g["n"], [[i, i, 1.0 + 0.1 * i] for i in range(g["n"])]), np.ones(g["n"]), g))
    g = golden["gmres_core_tridiag_6"]
    cases.append(("core_6", tridiag(g["n"], lo=-1.0, d=3.0, hi=-1.0), np.ones(g["n"]), g))
    return cases


def test_gmres_restart_ladder(oracle, golden):
    for requested, width in golden["gmres_restart_ladder"]["requested_width"]:
        assert oracle.gmres_width(requested) == width, requested


def test_gmres_golden(oracle, golden):
    g = golden["gmres_diagonal_2"]
    A = oracle.Csr.from_matrix(csr_from_lists(g["row_ptr"], g["col"], g["val"]))
    for _ in range(2):
        x, rep = oracle.gmres(A, np.array(g["b"]), restart=g["restart"], tol=g["tolerance"], rtol=0.0,
                              max_it=g["max_iterations"])
        assert rep.final_residual <= rep.threshold
        np.testing.assert_allclose(x, g["x"], atol=g["tol"])
    for name, M, b, g in gmres_golden_cases(golden):
        x, rep = oracle.gmres(oracle.Csr.from_matrix(M), b, restart=g["restart"], tol=g["tolerance"], rtol=0.0,
                              max_it=g["max_iterations"])
        assert rep.termination == "Converged", name
        assert np.linalg.norm(M.to_scipy() @ x - b) < g["residual_below"], name


def test_amg_gmres_golden(oracle, golden):
    """amg_integration_test.rs:125-142: AMG(default)-preconditioned GMRES(30)."""
    g = golden["amg_gmres_2d_16"]
    n = g["n"]
    A = grid_laplacian(n)
    xs = manufactured(n * n)
    Ao = oracle.Csr.from_matrix(A)
    x, rep = oracle.gmres(Ao, A.matvec(xs), restart=g["restart"], precond=oracle.PRE_AMG,
                          amg=oracle.Amg(Ao, oracle.AmgConfig()), tol=g["tolerance"], rtol=0.0,
                          max_it=g["max_iterations"])
    assert rep.termination == "Converged"
    assert np.max(np.abs(x - xs)) < g["max_abs_error"]


def test_gmres_against_scipy_and_history(oracle):
    """Nonsymmetric convection-diffusion-like tridiagonal system, Jacobi-right-
    preconditioned GMRES(8) with restarts: solution vs sparse direct, the
    implicit residual history is non-increasing within each run, and the
    budget ends in MaxIterations."""
    n = 300
    A = tridiag(n, lo=-1.3, d=3.0, hi=-0.7)
    b = np.random.default_rng(1).uniform(-1, 1, n)
    Ao = oracle.Csr.from_matrix(A)
    x, rep = oracle.gmres(Ao, b, restart=8, precond=oracle.PRE_JACOBI, rtol=1e-12, max_it=1000)
    assert rep.termination == "Converged" and rep.iterations > 8
    np.testing.assert_allclose(x, spla.spsolve(A.to_scipy().tocsc(), b), rtol=1e-9, atol=1e-10)
    h = rep.history
    assert np.all(np.diff(h) <= 1e-10 * h[0])  # GMRES never increases the residual
    _, rep = oracle.gmres(Ao, b, restart=8, precond=oracle.PRE_JACOBI, rtol=1e-14, max_it=5)
    assert rep.termination == "MaxIterations" and rep.iterations == 5
    _, rep = oracle.gmres(Ao, np.zeros(n), restart=8, rtol=1e-8)
    assert rep.termination == "InitialResidual" and rep.iterations == 0


def test_oracle_dense_coarse_solve_with_row_exchanges(oracle):
    """The oracle's dense coarsest solve (lu_factor / lu_solve) on matrices
    whose partial pivoting exchanges rows after the first columns (a Galerkin
    coarse operator that is not diagonally dominant, such as the 256^3
    constant-coefficient one, needs this): equal to numpy's solve. The row
    exchanges must all be applied to b before the forward substitution."""
    import numpy as np
    from cfdrs_b200.sparse import CsrMatrix
    rng = np.random.default_rng(4)
    for n in (6, 40, 120):
        M = rng.uniform(-1, 1, (n, n)) + np.diag(rng.uniform(0.05, 0.2, n))  # weak diagonal: many exchanges
        A = CsrMatrix.from_scipy(__import__("scipy.sparse", fromlist=["csr_matrix"]).csr_matrix(M))
        amg = oracle.Amg(oracle.Csr.from_matrix(A), oracle.AmgConfig(
            max_levels=1, min_coarse_size=4096, smoother=oracle.SMOOTH_JACOBI, coarse_solve=oracle.COARSE_DENSE))
        assert amg.num_levels == 1
        r = rng.uniform(-1, 1, n)
        z = amg.apply(r)
        ref = np.linalg.solve(M, r)
        assert np.linalg.norm(z - ref) <= 1e-10 * np.linalg.norm(ref), n
