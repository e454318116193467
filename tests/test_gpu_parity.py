"""GPU parity: the sm_100a path through the C ABI against the CPU oracle.

Tolerances (FP64 path): SpMV 1e-13 relative; hierarchy operators 1e-13;
V-cycle output 1e-11; Krylov solutions 1e-10 relative difference at an equal
residual tolerance with the same iteration count. FP32+refinement: solution
error <= 1e-8 against the FP64 oracle solution.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import csr_from_lists, grid_laplacian, manufactured, tridiag

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def dev(torch, a, dtype=None):
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda", dtype=dtype or torch.float64)


def random_csr(rng, n, ncols, lens):
    rp, col, val = [0], [], []
    for i in range(n):
        k = int(lens[i])
        cols = np.sort(rng.choice(ncols, size=min(k, ncols), replace=False))
        col += cols.tolist()
        val += rng.uniform(-1, 1, cols.size).tolist()
        rp.append(len(col))
    return csr_from_lists(rp, col, val, ncols)


def test_spmv_golden(cuda, golden):
    from cfdrs_b200.device import DeviceCsr
    g = golden["spmv_3x3"]
    A = DeviceCsr(csr_from_lists(g["row_ptr"], g["col"], g["val"]))
    x = dev(cuda, g["x"])
    y = cuda.zeros(3, device="cuda", dtype=cuda.float64)
    A.spmv(x.data_ptr(), y.data_ptr())
    cuda.cuda.synchronize()
    np.testing.assert_allclose(y.cpu().numpy(), g["y"], atol=g["tol"])


def spmv_case(shape):
    """Matrices of the SpMV parity tests; x-staged ones are marked True."""
    from cfdrs_b200 import problems as P
    rng = np.random.default_rng(7)
    staged = False
    if shape == "stencil":
        A, staged = P.poisson_3d_variable(20, 4.0, 1.0, seed=2)[0], True
    elif shape == "stencil_tail":  # 33^3 columns: the last x window ends in a 1-entry tail
        A, staged = P.poisson_3d_variable(33, 4.0, 1.0, seed=3)[0], True
    elif shape == "empty_blocks":  # > 2 blocks of empty rows between two stencils
        import scipy.sparse as sp
        from cfdrs_b200.sparse import CsrMatrix
        S = P.poisson_3d_fv(10)[0].to_scipy()
        A, staged = CsrMatrix.from_scipy(sp.block_diag([S, sp.csr_matrix((1300, 1300)), S]).tocsr()), True
    elif shape == "stencil_2d":  # the 2-D 128^2 operator: five diagonals
        A = P.poisson_2d_dirichlet(128, seed=0)[0]
    elif shape == "narrow":  # three columns: no bulk-copied window, all tail
        A, staged = random_csr(rng, 2000, 3, rng.integers(0, 4, 2000)), True
    elif shape == "ragged":  # empty rows and short rows of uneven length
        A = random_csr(rng, 3000, 3000, rng.integers(0, 12, 3000))
    elif shape == "long_rows":  # rows beyond the 2048-nonzero staging capacity
        lens = rng.integers(1, 20, 600)
        lens[[5, 300, 599]] = [2500, 4096, 3001]
        A = random_csr(rng, 600, 5000, lens)
    elif shape == "rectangular":
        A = random_csr(rng, 700, 1900, rng.integers(0, 30, 700))
    elif shape == "mixed":  # dictionary-coded stencil blocks followed by int32 random blocks
        import scipy.sparse as sp
        S1 = P.poisson_3d_fv(12)[0].to_scipy()
        S2 = random_csr(rng, 1500, S1.shape[1], rng.integers(0, 40, 1500)).to_scipy()
        from cfdrs_b200.sparse import CsrMatrix
        A = CsrMatrix.from_scipy(sp.vstack([S1, S2]).tocsr())
    elif shape == "coarse_operator_64":  # the 64^3 first coarse level: 23 diagonals, 2 threads per row
        import cfdrs_b200 as cf
        from cfdrs_b200.multigrid import HostHierarchy
        B = P.poisson_3d_variable(64, 8.0, 1.0, seed=0)[0]
        A, staged = HostHierarchy(B, cf.AMGConfig.pressure_poisson()).level(1, 0), False
    else:  # AMG operators of the 3-D solve: interpolation, restriction, coarse A (2 threads per row)
        import cfdrs_b200 as cf
        B = P.poisson_3d_variable(16, 4.0, 1.0, seed=2)[0]
        cfg = cf.AMGConfig.pressure_poisson()
        cfg.min_coarse_size = 100
        amg = cf.AlgebraicMultigrid(B, cfg)
        which = {"prolongation": (0, 1), "restriction": (0, 2), "coarse_operator": (1, 0)}[shape]
        A, staged = amg.level(*which), shape != "coarse_operator"
    return A, staged


@pytest.mark.parametrize("shape", ["stencil", "stencil_tail", "stencil_2d", "empty_blocks", "narrow", "ragged",
                                   "long_rows", "rectangular", "mixed", "prolongation", "restriction",
                                   "coarse_operator", "coarse_operator_64"])
def test_spmv_vs_oracle(cuda, oracle, shape):
    from cfdrs_b200.device import DeviceCsr
    A, staged = spmv_case(shape)
    rng = np.random.default_rng(11)
    x = rng.uniform(-1, 1, A.ncols)
    ref = oracle.Csr.from_matrix(A).spmv(x)
    d = DeviceCsr(A)
    y = cuda.zeros(A.nrows, device="cuda", dtype=cuda.float64)
    d.spmv(dev(cuda, x).data_ptr(), y.data_ptr())
    cuda.cuda.synchronize()
    np.testing.assert_allclose(y.cpu().numpy(), ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())
    y32 = cuda.zeros(A.nrows, device="cuda", dtype=cuda.float32)
    d.spmv(dev(cuda, x, cuda.float32).data_ptr(), y32.data_ptr(), fp32=True)
    cuda.cuda.synchronize()
    assert rel(y32.cpu().numpy().astype(np.float64), ref) < 1e-5
    if staged:
        assert d.layout()["x_staged"] == 1


@pytest.mark.parametrize("shape", ["stencil", "stencil_tail", "stencil_2d", "empty_blocks", "narrow",
                                   "prolongation", "restriction", "coarse_operator", "coarse_operator_64", "mixed"])
def test_spmv_pipelines_bit_identical(cuda, shape):
    """Every SpMV pipeline a matrix is eligible for (split, record, x-staged,
    diagonal, and for FP32 the sliced one) sums each row in the same order: FP64 and FP32
    results are bit-identical, and an x-staged request with an x that is not
    16-byte aligned runs on the record pipeline with the same result."""
    from cfdrs_b200.device import DeviceCsr
    A, staged = spmv_case(shape)
    d = DeviceCsr(A)
    lay = d.layout()
    if staged:
        assert lay["x_staged"] == 1
    paths = ["split"] + (["record"] if lay["all_compressed"] else []) + (["x_staged"] if lay["x_staged"] else []) + \
        (["diagonal"] if lay["diagonals"] else [])
    if shape in ("stencil", "stencil_tail", "stencil_2d"):
        assert lay["diagonals"] in (5, 7)
    if shape == "coarse_operator_64":
        assert lay["diagonals"] == 23 and lay["threads_per_row"] == 2
    x = np.random.default_rng(5).uniform(-1, 1, A.ncols)
    for dt in (cuda.float64, cuda.float32):
        fp32 = dt == cuda.float32
        xa = dev(cuda, x, dt)
        buf = cuda.zeros(A.ncols + 1, device="cuda", dtype=dt)
        buf[1:] = xa
        assert buf[1:].data_ptr() % 16 != 0
        ys = []
        for path in paths + (["sliced"] if fp32 and lay["sliced"] else []):
            d.set_path(path, fp32)
            for xp in ((xa, buf[1:]) if path == "x_staged" else (xa,)):
                y = cuda.full((A.nrows,), float("nan"), device="cuda", dtype=dt)
                d.spmv(xp.data_ptr(), y.data_ptr(), fp32=fp32)
                ys.append((path, y))
        cuda.cuda.synchronize()
        for path, y in ys[1:]:
            assert cuda.equal(ys[0][1], y), f"{shape} {dt} {path}"
        for mode in ("timed", "auto"):
            d.set_path(mode, fp32)
            y = cuda.zeros(A.nrows, device="cuda", dtype=dt)
            d.spmv(xa.data_ptr(), y.data_ptr(), fp32=fp32)  # "timed" keeps the fastest pipeline
            cuda.cuda.synchronize()
            assert cuda.equal(ys[0][1], y), f"{shape} {dt} {mode}"
            chosen = d.layout()["path_f32" if fp32 else "path_f64"]
            eligible = paths + (["sliced"] if fp32 and lay["sliced"] else [])
            assert chosen in [{"split": 0, "record": 1, "x_staged": 2, "sliced": 3, "diagonal": 4}[p] for p in eligible]
            if mode == "auto" and lay["diagonals"]:
                assert chosen == 4
            elif mode == "auto" and fp32:
                assert chosen == (1 if lay["all_compressed"] else 0)

@pytest.mark.parametrize("interp,order", [(0, 0), (2, 0), (2, 1)])
def test_amg_hierarchy_matches_oracle(cuda, oracle, interp, order):
    """Reference classical (0) / modified classical (2) interpolation, selection (0) /
    ascending (1) coarse numbering: the hierarchies agree level by level."""
    from cfdrs_b200 import problems as P
    from cfdrs_b200.multigrid import AlgebraicMultigrid, AMGConfig, InterpolationStrategy
    A = P.poisson_3d_variable(16, 4.0, 1.0, seed=5)[0]
    cfg = AMGConfig.pressure_poisson()
    cfg.min_coarse_size = 100
    cfg.interpolation_strategy = InterpolationStrategy(interp)
    cfg.coarse_order = order
    amg = AlgebraicMultigrid(A, cfg)
    ocfg = oracle.AmgConfig(max_levels=16, min_coarse_size=100, smoother=oracle.SMOOTH_JACOBI, pre_smooth=1,
                            post_smooth=1, relaxation=2 / 3, coarse_solve=oracle.COARSE_DENSE,
                            interpolation=interp, coarse_order=order)
    oamg = oracle.Amg(oracle.Csr.from_matrix(A), ocfg)
    assert amg.num_levels == oamg.num_levels >= 3
    for l in range(amg.num_levels):
        for which in (0, 1, 2):
            if which and l == amg.num_levels - 1:
                continue
            mine = amg.level(l, which)
            rp, ci, v, shape = oamg.level(l, which).arrays()
            assert mine.shape == shape
            np.testing.assert_array_equal(mine.row_ptr, rp)
            np.testing.assert_array_equal(mine.col, ci)
            np.testing.assert_allclose(mine.val, v, rtol=1e-13, atol=1e-13 * np.abs(v).max())


@pytest.mark.parametrize("coarse", ["dense", "sweeps"])
def test_vcycle_matches_oracle(cuda, oracle, coarse):
    from cfdrs_b200 import problems as P
    from cfdrs_b200.multigrid import AlgebraicMultigrid, AMGConfig, CoarseSolve
    A = P.poisson_3d_variable(16, 4.0, 1.0, seed=6)[0]
    cfg = AMGConfig.pressure_poisson()
    cfg.min_coarse_size = 100
    cfg.coarse_solve = CoarseSolve.DENSE if coarse == "dense" else CoarseSolve.SWEEPS
    amg = AlgebraicMultigrid(A, cfg)
    oamg = oracle.Amg(oracle.Csr.from_matrix(A), oracle.AmgConfig(
        max_levels=16, min_coarse_size=100, smoother=oracle.SMOOTH_JACOBI, pre_smooth=1, post_smooth=1,
        relaxation=2 / 3, coarse_solve=oracle.COARSE_DENSE if coarse == "dense" else oracle.COARSE_SWEEPS,
        interpolation=2, coarse_order=1))
    r = np.random.default_rng(1).uniform(-1, 1, A.nrows)
    z = amg.apply_to(r)
    assert rel(z, oamg.apply(r)) < 1e-11


def test_vcycle_bits_do_not_depend_on_the_pipeline(cuda):
    """One V-cycle (FP64, no dot products) gives the same bits whichever
    pipeline the operators run (the fine operator on the diagonal, record and
    split pipelines; every row sums in the same order on each)."""
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    A = P.poisson_3d_variable(24, 4.0, 1.0, seed=6)[0]
    cfg = cf.AMGConfig.pressure_poisson()
    cfg.min_coarse_size = 100
    amg = cf.AlgebraicMultigrid(A, cfg)
    r = np.random.default_rng(3).uniform(-1, 1, A.nrows)
    zs = []
    for path in ("diagonal", "record", "split", "auto"):
        amg.set_path(path, False)
        zs.append(amg.apply_to(r))
    amg.set_path("auto", False)
    for z in zs[1:]:
        assert np.array_equal(z.view(np.int64), zs[0].view(np.int64))


def _oracle_solve(oracle, A, b, pre, solver="pcg", amg=None, rtol=1e-8, max_it=5000):
    Ao = oracle.Csr.from_matrix(A)
    return getattr(oracle, solver)(Ao, b, precond=pre, amg=amg, rtol=rtol, max_it=max_it)


def test_pcg_jacobi_c1_parity(cuda, oracle):
    """2-D pressure Poisson 128x128, Jacobi-PCG to 1e-8 (the CPU-runnable case)."""
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    A, b = P.poisson_2d_dirichlet(128, seed=0)
    xo, ro = _oracle_solve(oracle, A, b, oracle.PRE_JACOBI)
    x = np.zeros_like(b)
    rep = cf.cg_preconditioned(A, b, cf.JacobiPreconditioner(A), x,
                               cf.IterativeSolverConfig(0.0, 1e-8, 5000))
    assert rep.termination == cf.Termination.CONVERGED and ro.termination == "Converged"
    assert abs(rep.iterations - ro.iterations) <= 1
    assert rel(x, xo) < 1e-10
    assert np.linalg.norm(b - A.matvec(x)) <= 1.0000001e-8 * np.linalg.norm(b)


@pytest.mark.parametrize("pre", ["jacobi", "none"])
def test_cluster_solve_matches_multi_kernel_solve(cuda, oracle, pre):
    """Small systems run CG / Jacobi-PCG as one thread-block-cluster launch:
    the 128^2 pressure system (16 384 rows) gives the multi-kernel solve's
    iteration count to one and its solution to 1e-10, with a single kernel
    launch; a 256^2 system does not fit a cluster's shared memory and runs
    the multi-kernel solve."""
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.device import device_matrix
    A, b = P.poisson_2d_dirichlet(128, seed=0)
    dm = device_matrix(A)
    pc = cf.JacobiPreconditioner(A) if pre == "jacobi" else None
    cfgs = cf.IterativeSolverConfig(0.0, 1e-8, 5000)

    def solve(cluster):
        dm.ctx.set_cluster_solve(cluster)
        x = np.zeros_like(b)
        rep = cf.cg_preconditioned(A, b, pc, x, cfgs) if pc is not None else cf.cg(A, b, x, cfgs)
        return x, rep, dm.ctx.kernel_stats()["launches"]
    try:
        x1, r1, l1 = solve(True)
        x2, r2, l2 = solve(False)
    finally:
        dm.ctx.set_cluster_solve(True)
    assert r1.termination == r2.termination == cf.Termination.CONVERGED
    assert abs(r1.iterations - r2.iterations) <= 1 and l1 == 1 and l2 > 3 * r2.iterations
    assert rel(x1, x2) < 1e-10
    assert abs(r1.initial_residual_norm - r2.initial_residual_norm) <= 1e-13 * r2.initial_residual_norm
    opre = oracle.PRE_JACOBI if pre == "jacobi" else oracle.PRE_NONE
    xo, ro = _oracle_solve(oracle, A, b, opre)
    assert abs(r1.iterations - ro.iterations) <= 1 and rel(x1, xo) < 1e-10
    B, bb = P.poisson_2d_dirichlet(256, seed=0)
    xb = np.zeros_like(bb)
    rb = cf.cg_preconditioned(B, bb, cf.JacobiPreconditioner(B), xb, cfgs)
    assert rb.termination == cf.Termination.CONVERGED and device_matrix(B).ctx.kernel_stats()["launches"] > 3


def test_cluster_solve_edge_cases(cuda):
    """Fewer rows than the cluster's CTAs could hold (17 rows over two CTAs,
    an odd split), a warm start at the solution, and the iteration budget."""
    import cfdrs_b200 as cf
    A = tridiag(17, lo=-1.0, d=2.5, hi=-1.0)
    b = np.random.default_rng(4).uniform(-1, 1, 17)
    x = np.zeros(17)
    rep = cf.cg_preconditioned(A, b, cf.JacobiPreconditioner(A), x, cf.IterativeSolverConfig(0.0, 1e-12, 100))
    assert rep.termination == cf.Termination.CONVERGED
    np.testing.assert_allclose(A.matvec(x), b, atol=1e-10)
    rep = cf.cg_preconditioned(A, b, cf.JacobiPreconditioner(A), x.copy(), cf.IterativeSolverConfig(1e-6, 0.0, 100))
    assert rep.termination == cf.Termination.INITIAL_RESIDUAL and rep.iterations == 0
    rep = cf.cg(A, b, np.zeros(17), cf.IterativeSolverConfig(0.0, 1e-14, 3))
    assert rep.termination == cf.Termination.MAX_ITERATIONS and rep.iterations == 3


def test_amg_pcg_parity(cuda, oracle):
    """3-D Poisson (constant k), AMG-PCG V(1,1) Jacobi w=2/3, dense coarsest, to 1e-8."""
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    A, b = P.poisson_3d_fv(32, seed=1)
    cfg = cf.AMGConfig.pressure_poisson()
    cfg.min_coarse_size = 512
    amg = cf.AlgebraicMultigrid(A, cfg)
    oamg = oracle.Amg(oracle.Csr.from_matrix(A), oracle.AmgConfig(
        max_levels=16, min_coarse_size=512, smoother=oracle.SMOOTH_JACOBI, pre_smooth=1, post_smooth=1,
        relaxation=2 / 3, coarse_solve=oracle.COARSE_DENSE, interpolation=2, coarse_order=1))
    xo, ro = _oracle_solve(oracle, A, b, oracle.PRE_AMG, amg=oamg)
    x = np.zeros_like(b)
    rep = cf.cg_preconditioned(A, b, amg, x, cf.IterativeSolverConfig(0.0, 1e-8, 500))
    assert rep.termination == cf.Termination.CONVERGED
    assert rep.iterations == ro.iterations
    assert rel(x, xo) < 1e-10


@pytest.mark.parametrize("pre", ["none", "jacobi", "amg"])
def test_bicgstab_parity(cuda, oracle, pre):
    import cfdrs_b200 as cf
    if pre == "amg":
        A = grid_laplacian(24)
        b = A.matvec(manufactured(A.nrows))
    else:
        A = tridiag(400, lo=-1.3, d=3.0, hi=-0.7)
        b = np.random.default_rng(3).uniform(-1, 1, 400)
    amg = oamg = None
    if pre == "amg":
        cfg = cf.AMGConfig(pre_smooth_iterations=1, post_smooth_iterations=1, relaxation_factor=2 / 3)
        amg = cf.AlgebraicMultigrid(A, cfg)
        oamg = oracle.Amg(oracle.Csr.from_matrix(A), oracle.AmgConfig(
            smoother=oracle.SMOOTH_JACOBI, pre_smooth=1, post_smooth=1, relaxation=2 / 3))
        P_ = amg
    else:
        P_ = cf.JacobiPreconditioner(A) if pre == "jacobi" else None
    opre = {"none": oracle.PRE_NONE, "jacobi": oracle.PRE_JACOBI, "amg": oracle.PRE_AMG}[pre]
    xo, ro = _oracle_solve(oracle, A, b, opre, solver="bicgstab", amg=oamg, rtol=1e-10)
    x = np.zeros_like(b)
    cfgs = cf.IterativeSolverConfig(0.0, 1e-10, 500)
    rep = (cf.bicgstab_preconditioned(A, b, P_, x, cfgs) if P_ is not None else cf.bicgstab(A, b, x, cfgs))
    assert rep.termination == cf.Termination.CONVERGED and ro.termination == "Converged"
    assert abs(rep.iterations - ro.iterations) <= 1
    assert rel(x, xo) < 1e-9


@pytest.mark.parametrize("solver", ["cg", "bicgstab"])
def test_diagonal_golden_gpu(cuda, golden, solver):
    import cfdrs_b200 as cf
    g = golden["diagonal_solve_2"]
    A = csr_from_lists(g["row_ptr"], g["col"], g["val"])
    for _ in range(2):
        x = np.zeros(2)
        fn = cf.cg if solver == "cg" else cf.bicgstab
        rep = fn(A, np.array(g["b"]), x, cf.IterativeSolverConfig(g["tolerance"], 0.0, g["max_iterations"]))
        assert rep.final_residual_norm <= rep.threshold
        np.testing.assert_allclose(x, g["x"], atol=g["tol"])


def test_amg_integration_gpu(cuda, golden):
    """amg_integration_test.rs:97-122 on the device V-cycle (damped Jacobi smoother)."""
    import cfdrs_b200 as cf
    g = golden["amg_poisson_2d_16"]
    A = grid_laplacian(g["n"])
    xs = manufactured(A.nrows)
    b = A.matvec(xs)
    amg = cf.AlgebraicMultigrid(A, cf.AMGConfig(relaxation_factor=2 / 3))
    for fn in (cf.bicgstab_preconditioned, cf.cg_preconditioned):
        x = np.zeros_like(b)
        rep = fn(A, b, amg, x, cf.IterativeSolverConfig(g["tolerance"], 0.0, g["max_iterations"]))
        assert rep.termination == cf.Termination.CONVERGED
        assert np.max(np.abs(x - xs)) < g["max_abs_error"]


@pytest.mark.parametrize("solver", ["cg", "bicgstab"])
def test_fp32_refinement_error(cuda, oracle, solver):
    """FP32 inner AMG Krylov + FP64 refinement to 1e-10: error vs the FP64 oracle <= 1e-8."""
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    A, b, _ = P.poisson_3d_variable(32, 8.0, 1.0, seed=0)
    cfg = cf.AMGConfig.pressure_poisson()
    cfg.min_coarse_size = 512
    amg = cf.AlgebraicMultigrid(A, cfg)
    oamg = oracle.Amg(oracle.Csr.from_matrix(A), oracle.AmgConfig(
        max_levels=16, min_coarse_size=512, smoother=oracle.SMOOTH_JACOBI, pre_smooth=1, post_smooth=1,
        relaxation=2 / 3, coarse_solve=oracle.COARSE_DENSE, interpolation=2, coarse_order=1))
    xo, ro = _oracle_solve(oracle, A, b, oracle.PRE_AMG, amg=oamg, rtol=1e-13, max_it=500)
    x = np.zeros_like(b)
    fn = cf.cg_preconditioned if solver == "cg" else cf.bicgstab_preconditioned
    rep = fn(A, b, amg, x, cf.IterativeSolverConfig(0.0, 1e-10, 500), precision=cf.Precision.FP32_REFINE)
    assert rep.termination == cf.Termination.CONVERGED
    assert rep.outer_iterations >= 2
    true_res = np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b)
    assert true_res <= 1e-10 * 1.0001
    assert rel(x, xo) <= 1e-8


def test_device_pointer_solve_matches_host(cuda):
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    A, b = P.poisson_2d_dirichlet(48, seed=9)
    x_host = np.zeros_like(b)
    cfgs = cf.IterativeSolverConfig(0.0, 1e-9, 2000)
    r1 = cf.cg_preconditioned(A, b, cf.JacobiPreconditioner(A), x_host, cfgs)
    bd = dev(cuda, b)
    xd = cuda.zeros_like(bd)
    r2 = cf.cg_preconditioned(A, bd, cf.JacobiPreconditioner(A), xd, cfgs)
    assert r1.iterations == r2.iterations
    np.testing.assert_array_equal(xd.cpu().numpy(), x_host)


def test_termination_and_errors(cuda):
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    A, b = P.poisson_2d_dirichlet(16, seed=1)
    J = cf.JacobiPreconditioner(A)
    rep = cf.cg_preconditioned(A, b, J, np.zeros_like(b), cf.IterativeSolverConfig(0.0, 1e-12, 1))
    assert rep.termination == cf.Termination.MAX_ITERATIONS and rep.iterations == 1
    assert cf.interpret("t", rep).kind == cf.SolveOutcome.STALLED
    rep = cf.cg_preconditioned(A, np.zeros_like(b), J, np.zeros_like(b), cf.IterativeSolverConfig(0.0, 1e-8, 10))
    assert rep.termination == cf.Termination.INITIAL_RESIDUAL and rep.iterations == 0
    neg = csr_from_lists([0, 1, 2], [0, 1], [-1.0, -2.0])
    rep = cf.cg(neg, np.ones(2), np.zeros(2), cf.IterativeSolverConfig(0.0, 1e-8, 10))
    assert rep.termination == cf.Termination.NON_POSITIVE_CURVATURE
    assert cf.interpret("t", rep).kind == cf.SolveOutcome.BROKEN_DOWN
    with pytest.raises(cf.SolveError):
        cf.cg(A, b[:-1], np.zeros(A.nrows), cf.IterativeSolverConfig(0.0, 1e-8, 10))
    with pytest.raises(cf.SolveError):
        cf.cg(A, b, np.zeros_like(b), cf.IterativeSolverConfig(0.0, 1e-8, 0))
    bad = csr_from_lists([0, 1, 2], [0, 1], [np.inf, 1.0])
    with pytest.raises(cf.SolveError, match="NONFINITE"):
        cf.cg_preconditioned(bad, np.ones(2), cf.JacobiPreconditioner(bad), np.zeros(2),
                             cf.IterativeSolverConfig(0.0, 1e-8, 10))
    x = np.zeros(2)
    rep = cf.cg(csr_from_lists([0, 1, 2], [0, 1], [1.0, 1.0]), np.array([np.nan, 1.0]), x,
                cf.IterativeSolverConfig(0.0, 1e-8, 10))
    assert rep.termination == cf.Termination.BREAKDOWN


def test_recompute_matches_fresh_setup(cuda):
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    A1 = P.poisson_3d_variable(12, 3.0, 1.0, seed=1)[0]
    A2 = P.poisson_3d_variable(12, 3.0, 1.0, seed=2)[0]
    cfg = cf.AMGConfig.pressure_poisson()
    cfg.min_coarse_size = 64
    amg = cf.AlgebraicMultigrid(A1, cfg)
    amg.recompute(A2)
    fresh_P = cf.AlgebraicMultigrid(A1.with_values(A1.val), cfg)
    r = np.random.default_rng(0).uniform(-1, 1, A1.nrows)
    z = amg.apply_to(r)
    # recompute keeps the transfer operators of A1 and re-forms the Galerkin chain of A2
    np.testing.assert_array_equal(amg.level(0, 1).val, fresh_P.level(0, 1).val)
    np.testing.assert_allclose(amg.level(0, 0).val, A2.val)
    assert np.all(np.isfinite(z))


def test_solve_on_every_pipeline(cuda):
    """The AMG-PCG solve (FP64 and FP32 + refinement) converges to the same
    solution whichever SpMV pipeline the operators run. Row products are
    identical; the fused dot products sum their per-CTA partials over each
    pipeline's own grid, so iterates agree to rounding, not bit for bit."""
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.device import device_matrix
    A, b, _ = P.poisson_3d_variable(24, 8.0, 1.0, seed=1)
    cfg = cf.AMGConfig.pressure_poisson()
    cfg.min_coarse_size = 200
    amg = cf.AlgebraicMultigrid(A, cfg)
    dA = device_matrix(A)
    bd = dev(cuda, b)
    conf = cf.IterativeSolverConfig(0.0, 1e-10, 500)
    for prec in (cf.Precision.FP64, cf.Precision.FP32_REFINE):
        fp32 = prec == cf.Precision.FP32_REFINE
        xs = []
        assert dA.layout()["diagonals"] == 7
        for path in ("auto", "split", "record", "x_staged", "diagonal", "timed"):
            amg.set_path(path, fp32)
            try:
                dA.set_path(path, fp32)
            except Exception:
                dA.set_path("auto", fp32)
            x = cuda.zeros_like(bd)
            rep = cf.cg_preconditioned(A, bd, amg, x, conf, precision=prec)
            assert rep.termination == cf.Termination.CONVERGED
            xs.append((x.cpu().numpy(), rep.iterations))
        amg.set_path("auto", fp32)
        dA.set_path("auto", fp32)
        x0, it0 = xs[0]
        for x, it in xs[1:]:
            assert abs(it - it0) <= 1, prec
            assert rel(x, x0) < 1e-8, prec
