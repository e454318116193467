"""Adjoint of the device solve (SparseSolveFunction): pattern outer product,
gradients with respect to values and right-hand side, and dL/dtheta of the 2-D
Darcy column loss against the CPU FP64 adjoint and central differences.

Tolerances: pattern outer product 1e-15 relative; value/rhs gradients 1e-9
(FP64 Jacobi-PCG to 1e-13 vs direct); dL/dtheta (forward and adjoint FP32 +
FP64 refinement to 1e-10) within 1e-6 (2-norm, relative) of the CPU adjoint and
within 1e-5 of max |g| of central differences (h = 1e-6) on 64 seeded cells.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_pattern_outer(cuda):
    torch = cuda
    from cfdrs_b200 import problems as P
    from cfdrs_b200.adjoint import SparseSolver
    A, _ = P.poisson_2d_dirichlet(20)
    s = SparseSolver(A, preconditioner="jacobi")
    rng = np.random.default_rng(0)
    lam, x = rng.standard_normal(A.nrows), rng.standard_normal(A.nrows)
    g = s.pattern_outer(torch.as_tensor(lam, device="cuda"), torch.as_tensor(x, device="cuda"), 2.0)
    rows = np.repeat(np.arange(A.nrows), np.diff(A.row_ptr))
    np.testing.assert_allclose(g.cpu().numpy(), -2.0 * lam[rows] * x[A.col], rtol=1e-15)


def test_sparse_solve_gradients(cuda):
    torch = cuda
    import scipy.sparse.linalg as spla
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.adjoint import SparseSolver, sparse_solve
    theta = P.gaussian_random_field((24, 24), 3.0, 0.5, seed=1)
    A, b = P.darcy_2d(theta)
    s = SparseSolver(A, preconditioner="jacobi", precision=cf.Precision.FP64,
                     config=cf.IterativeSolverConfig(0.0, 1e-13, 5000))
    vals = torch.as_tensor(np.array(A.val), device="cuda").requires_grad_(True)
    bt = torch.as_tensor(b, device="cuda").requires_grad_(True)
    w = torch.as_tensor(np.random.default_rng(2).standard_normal(A.nrows), device="cuda")
    x = sparse_solve(vals, bt, s)
    (x * w).sum().backward()
    S = A.to_scipy().tocsc()
    xs = spla.spsolve(S, b)
    lam = spla.spsolve(S.T.tocsc(), w.cpu().numpy())
    rows = np.repeat(np.arange(A.nrows), np.diff(A.row_ptr))
    np.testing.assert_allclose(x.detach().cpu().numpy(), xs, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(bt.grad.cpu().numpy(), lam, rtol=1e-9, atol=1e-12 * np.abs(lam).max())
    gv = -lam[rows] * xs[A.col]
    np.testing.assert_allclose(vals.grad.cpu().numpy(), gv, rtol=1e-8, atol=1e-10 * np.abs(gv).max())


def test_darcy_theta_gradient_vs_cpu_adjoint_and_fd(cuda):
    torch = cuda
    import adjoint_cpu as AC
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.adjoint import (SparseSolver, column_loss, darcy_2d_pattern, darcy_2d_torch,
                                    loss_column_index, sparse_solve)
    n = 128
    theta = P.gaussian_random_field((n, n), 4.0, 0.5, seed=7)
    col = loss_column_index(n)
    pattern, mask = darcy_2d_pattern(n)
    cfg = cf.AMGConfig.pressure_poisson()
    cfg.min_coarse_size = 1024
    s = SparseSolver(pattern, amg_config=cfg, precision=cf.Precision.FP32_REFINE,
                     config=cf.IterativeSolverConfig(0.0, 1e-10, 500))
    th = torch.as_tensor(theta, device="cuda").requires_grad_(True)
    vals, b = darcy_2d_torch(th, torch.as_tensor(mask, device="cuda"))
    p = sparse_solve(vals, b, s, True)
    L = column_loss(p, n, col)
    L.backward()
    g = th.grad.cpu().numpy()
    L_cpu, g_cpu, _ = AC.loss_and_grad(theta, col)
    assert abs(L.item() - L_cpu) <= 1e-9 * abs(L_cpu)
    assert np.linalg.norm(g - g_cpu) <= 1e-6 * np.linalg.norm(g_cpu)
    rng = np.random.default_rng(64)
    cells = [(int(j), int(i)) for j, i in rng.integers(0, n, size=(64, 2))]
    fd = AC.central_fd(theta, col, cells, h=1e-6)
    ga = np.array([g[j, i] for j, i in cells])
    assert np.abs(ga - fd).max() <= 1e-5 * np.abs(g_cpu).max()


def test_darcy_512_gradient_vs_cpu_adjoint_and_fd(cuda):
    """The adjoint workload at full size (512^2 cells, theta GRF l = 16,
    sigma = 0.5, forward and adjoint FP32 + FP64 refinement to 1e-10): the
    device gradient against the FP64 CPU adjoint, and both against central
    differences (h = 1e-6, FP64) on the 64 seeded cells of the configuration.
    Every perturbed system is solved from one sparse LU of the unperturbed
    matrix by the Woodbury identity (adjoint_cpu.central_fd_lowrank): exact
    algebra, and the rounding of a single factorization cancels in the
    difference, so the FD noise is about 1.5e-5 max|g| at kappa ~ 1e6 instead
    of the 3e-4 of two independent factorizations per cell."""
    torch = cuda
    import adjoint_cpu as AC
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.adjoint import (SparseSolver, column_loss, darcy_2d_pattern, darcy_2d_torch,
                                    loss_column_index, sparse_solve)
    n = 512
    theta = P.gaussian_random_field((n, n), 16.0, 0.5, seed=0)
    col = loss_column_index(n)
    pattern, mask = darcy_2d_pattern(n)
    s = SparseSolver(pattern, precision=cf.Precision.FP32_REFINE, config=cf.IterativeSolverConfig(0.0, 1e-10, 500))
    th = torch.as_tensor(theta, device="cuda").requires_grad_(True)
    vals, b = darcy_2d_torch(th, torch.as_tensor(mask, device="cuda"))
    L = column_loss(sparse_solve(vals, b, s, True), n, col)
    L.backward()
    g = th.grad.cpu().numpy()
    L_cpu, g_cpu, _ = AC.loss_and_grad(theta, col)
    assert abs(L.item() - L_cpu) <= 1e-9 * abs(L_cpu)
    assert np.linalg.norm(g - g_cpu) <= 1e-8 * np.linalg.norm(g_cpu)
    rng = np.random.default_rng(64)
    cells = [(int(j), int(i)) for j, i in rng.integers(0, n, size=(64, 2))]
    fd = AC.central_fd_lowrank(theta, col, cells, h=1e-6)
    ga = np.array([g[j, i] for j, i in cells])
    gc = np.array([g_cpu[j, i] for j, i in cells])
    scale = np.abs(g_cpu).max()
    assert np.abs(ga - fd).max() <= 1e-4 * scale
    assert np.abs(ga - fd).max() <= 2.0 * np.abs(gc - fd).max() + 1e-9 * scale  # no worse than the CPU adjoint


@pytest.mark.parametrize("n", [1, 2, 37, 64])
def test_darcy_assembly_kernel_equals_torch_assembly(cuda, n):
    """cfd_darcy2d_assemble performs the torch assembly's operations in its
    order: values and right-hand side equal bit for bit (1 x 1 and 2 x 2
    grids included: both walls on one cell)."""
    torch = cuda
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.adjoint import SparseSolver, darcy_2d_assemble_device, darcy_2d_pattern, darcy_2d_torch
    theta = P.gaussian_random_field((n, n), 4.0, 0.5, seed=n) if n > 2 else \
        np.random.default_rng(n).standard_normal((n, n))
    pattern, mask = darcy_2d_pattern(n)
    s = SparseSolver(pattern, preconditioner="jacobi", precision=cf.Precision.FP64)
    th = torch.as_tensor(theta, device="cuda")
    v_t, b_t = darcy_2d_torch(th, torch.as_tensor(mask, device="cuda"))
    v_d, b_d = darcy_2d_assemble_device(th, s)
    assert torch.equal(v_t, v_d) and torch.equal(b_t, b_d)
    A, b = P.darcy_2d(theta)  # the scipy assembly of the same system
    np.testing.assert_allclose(v_d.cpu().numpy(), A.val, rtol=1e-14)
    np.testing.assert_allclose(b_d.cpu().numpy(), b, rtol=1e-14)


def test_darcy_kernels_refuse_other_patterns(cuda):
    torch = cuda
    import cfdrs_b200 as cf
    from cfdrs_b200 import _lib
    from cfdrs_b200 import problems as P
    from cfdrs_b200.adjoint import SparseSolver, darcy_2d_assemble_device
    import scipy.sparse as sp
    from cfdrs_b200.sparse import CsrMatrix
    # 256 rows but a 9-point pattern
    S = sp.diags([1.0] * 9, [-17, -16, -15, -1, 0, 1, 15, 16, 17], shape=(256, 256)).tocsr()
    A = CsrMatrix(S.indptr.astype(np.int64), S.indices.astype(np.int64), S.data, S.shape)
    s = SparseSolver(A, preconditioner="jacobi", precision=cf.Precision.FP64)
    with pytest.raises(_lib.CfdError, match="Darcy pattern") as e:
        darcy_2d_assemble_device(torch.zeros((16, 16), dtype=torch.float64, device="cuda"), s)
    assert e.value.status == 1
    # the 5-point pattern of a 16 x 16 grid is that pattern; a 15 x 15 theta does not fit it
    A5, _ = P.poisson_2d_dirichlet(16)
    s5 = SparseSolver(A5, preconditioner="jacobi", precision=cf.Precision.FP64)
    darcy_2d_assemble_device(torch.zeros((16, 16), dtype=torch.float64, device="cuda"), s5)
    with pytest.raises(_lib.CfdError, match="Darcy pattern"):
        darcy_2d_assemble_device(torch.zeros((15, 15), dtype=torch.float64, device="cuda"), s5)


def test_darcy_512_fused_gradient(cuda):
    """The adjoint workload through DarcySolveFunction (assembly and chain
    rule each one kernel): loss and dL/dtheta equal the generic path's
    (torch assembly, SparseSolveFunction, autograd) to 1e-10 and the FP64 CPU
    adjoint's to 1e-8; on the 64 seeded cells within 1e-4 max|g| of central
    differences (h = 1e-6, low-rank exact perturbed solves)."""
    torch = cuda
    import adjoint_cpu as AC
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.adjoint import (SparseSolver, column_loss, darcy_2d_pattern, darcy_2d_solve, darcy_2d_torch,
                                    loss_column_index, sparse_solve)
    n = 512
    theta = P.gaussian_random_field((n, n), 16.0, 0.5, seed=0)
    col = loss_column_index(n)
    pattern, mask = darcy_2d_pattern(n)
    cfg = cf.IterativeSolverConfig(0.0, 1e-10, 500)
    s = SparseSolver(pattern, precision=cf.Precision.FP32_REFINE, config=cfg)
    th = torch.as_tensor(theta, device="cuda").requires_grad_(True)
    L = column_loss(darcy_2d_solve(th, s, True), n, col)
    L.backward()
    g = th.grad.cpu().numpy()
    s2 = SparseSolver(pattern, precision=cf.Precision.FP32_REFINE, config=cfg)
    th2 = torch.as_tensor(theta, device="cuda").requires_grad_(True)
    vals, b = darcy_2d_torch(th2, torch.as_tensor(mask, device="cuda"))
    L2 = column_loss(sparse_solve(vals, b, s2, True), n, col)
    L2.backward()
    g2 = th2.grad.cpu().numpy()
    assert abs(L.item() - L2.item()) <= 1e-12 * abs(L2.item())
    assert np.linalg.norm(g - g2) <= 1e-10 * np.linalg.norm(g2)
    L_cpu, g_cpu, _ = AC.loss_and_grad(theta, col)
    assert abs(L.item() - L_cpu) <= 1e-9 * abs(L_cpu)
    assert np.linalg.norm(g - g_cpu) <= 1e-8 * np.linalg.norm(g_cpu)
    rng = np.random.default_rng(64)
    cells = [(int(j), int(i)) for j, i in rng.integers(0, n, size=(64, 2))]
    fd = AC.central_fd_lowrank(theta, col, cells, h=1e-6)
    ga = np.array([g[j, i] for j, i in cells])
    assert np.abs(ga - fd).max() <= 1e-4 * np.abs(g_cpu).max()


@pytest.mark.parametrize("precision", ["fp64", "fp32_refine"])
def test_nonsymmetric_adjoint_is_a_transposed_solve(cuda, precision):
    """A non-symmetric operator (diffusion plus first-order upwind convection
    on 24 x 24 cells): the backward solves A^T lambda = dL/dx on A's
    transpose (cfd_adjoint, BiCGSTAB with Jacobi), so dL/db = A^-T w and
    dL/dA = -lambda x^T on the pattern match the direct solves to 1e-8; a
    value update re-forms the transpose."""
    torch = cuda
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    import cfdrs_b200 as cf
    from cfdrs_b200.adjoint import SparseSolver, sparse_solve
    from cfdrs_b200.sparse import CsrMatrix
    n = 24
    e = np.ones(n)
    T = sp.diags([-e[:-1], 2 * e, -e[:-1]], [-1, 0, 1])
    U = sp.diags([-e[:-1], e], [-1, 0])  # upwind first difference
    I = sp.identity(n)
    S = (sp.kron(I, T) + sp.kron(T, I) + 0.8 * sp.kron(I, U)).tocsr()
    S.sort_indices()
    A = CsrMatrix(S.indptr.astype(np.int64), S.indices.astype(np.int64), S.data.copy(), S.shape)
    prec = cf.Precision.FP64 if precision == "fp64" else cf.Precision.FP32_REFINE
    s = SparseSolver(A, preconditioner="jacobi", solver="bicgstab", precision=prec,
                     config=cf.IterativeSolverConfig(0.0, 1e-13 if precision == "fp64" else 1e-11, 5000))
    rng = np.random.default_rng(5)
    b = rng.standard_normal(n * n)
    w = torch.as_tensor(rng.standard_normal(n * n), device="cuda")
    rows = np.repeat(np.arange(n * n), np.diff(A.row_ptr))
    for scale in (1.0, 1.7):
        vals = torch.as_tensor(scale * A.val, device="cuda").requires_grad_(True)
        bt = torch.as_tensor(b, device="cuda").requires_grad_(True)
        x = sparse_solve(vals, bt, s)
        assert s.symmetric is False
        (x * w).sum().backward()
        Sc = (scale * S).tocsc()
        xs = spla.spsolve(Sc, b)
        lam = spla.spsolve(Sc.T.tocsc(), w.cpu().numpy())
        tol = 1e-8 if precision == "fp64" else 1e-7
        assert np.linalg.norm(bt.grad.cpu().numpy() - lam) <= tol * np.linalg.norm(lam)
        gv = -lam[rows] * xs[A.col]
        assert np.linalg.norm(vals.grad.cpu().numpy() - gv) <= tol * np.linalg.norm(gv)
