"""GMRES + SIMPLE and GMRES + block diagonal on the device (the saddle-point
tiers of LinearSolverChain, chain.rs:216-238, 265-285), against the host path
of the same preconditioner code (bit for bit) and the oracle's GMRES with the
same preconditioner (iterations within 10 % + 5,
error against the direct solution within 10x the oracle's own, or 1e-9
relative; FP32 inside FP64 refinement: error <= 1e-8 relative)."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

pytestmark = pytest.mark.gpu


def same_bits(a, b):
    return a.shape == b.shape and np.array_equal(np.ascontiguousarray(a).view(np.int64),
                                                 np.ascontiguousarray(b).view(np.int64))


@pytest.mark.parametrize("n", [8, 24])
def test_device_apply_equals_host(cuda, n):
    import torch
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.saddle import simple_apply_host
    A, b, nv = P.stokes_2d_mac(n)
    M = cf.SimplePreconditioner(A, nv)
    r = np.random.default_rng(n).standard_normal(A.shape[0])
    z = M.apply(torch.tensor(r, device="cuda")).cpu().numpy()
    assert same_bits(z, simple_apply_host(A, nv, r))


@pytest.mark.parametrize("n", [16, 32])
def test_gmres_simple_matches_oracle(cuda, oracle, n):
    import torch
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    A, b, nv = P.stokes_2d_mac(n)
    x_ref = spla.spsolve(A.to_scipy().tocsc(), b)
    Ao = oracle.Csr.from_matrix(A)
    xo, ro = oracle.gmres_simple(Ao, oracle.Simple(Ao, nv), b, restart=30, rtol=1e-10, max_it=20000)
    M = cf.SimplePreconditioner(A, nv)
    cfg = cf.IterativeSolverConfig(0.0, 1e-10, 20000)
    x = np.zeros(A.shape[0])
    rep = cf.gmres_preconditioned(A, b, M, x, cfg, restart=30)
    assert rep.termination == cf.Termination.CONVERGED
    assert abs(rep.iterations - ro.iterations) <= 0.10 * ro.iterations + 5, (rep.iterations, ro.iterations)
    err, err_o = np.linalg.norm(x - x_ref), np.linalg.norm(xo - x_ref)
    assert err <= max(10 * err_o, 1e-9 * np.linalg.norm(x_ref)), (err, err_o)
    xd = torch.zeros(A.shape[0], dtype=torch.float64, device="cuda")
    rep32 = cf.gmres_preconditioned(A, torch.tensor(b, device="cuda"), M, xd, cfg, restart=30,
                                    precision=cf.Precision.FP32_REFINE)
    assert rep32.termination == cf.Termination.CONVERGED
    assert np.linalg.norm(xd.cpu().numpy() - x_ref) <= 1e-8 * np.linalg.norm(x_ref)


def test_simple_rules_and_value_updates(cuda):
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.krylov import SolveError
    from cfdrs_b200.device import device_matrix
    A, b, nv = P.stokes_2d_mac(12)
    M = cf.SimplePreconditioner(A, nv)
    cfg = cf.IterativeSolverConfig(0.0, 1e-10, 20000)
    with pytest.raises(SolveError, match="GMRES only"):
        cf.cg_preconditioned(A, b, M, np.zeros(A.shape[0]), cfg)
    with pytest.raises(SolveError, match="another matrix"):
        cf.gmres_preconditioned(A.with_values(A.val.copy()), b, M, np.zeros(A.shape[0]), cfg)
    x1 = np.zeros(A.shape[0])
    cf.gmres_preconditioned(A, b, M, x1, cfg, restart=30)
    # new values on the same pattern: the SIMPLE arrays are rebuilt before the next solve
    device_matrix(A).update_values(2.0 * A.val)
    x2 = np.zeros(A.shape[0])
    rep = cf.gmres_preconditioned(A, b, M, x2, cfg, restart=30)
    assert rep.termination == cf.Termination.CONVERGED
    assert np.linalg.norm(2.0 * x2 - x1) <= 1e-8 * np.linalg.norm(x1)


def test_block_diagonal_device(cuda, oracle):
    import torch
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.saddle import block_diagonal_host
    A, b, nv = P.stokes_2d_mac(16)
    M = cf.BlockDiagonalPreconditioner(A, nv)
    r = np.random.default_rng(3).standard_normal(A.shape[0])
    z = M.apply(torch.tensor(r, device="cuda")).cpu().numpy()
    assert same_bits(z, r * block_diagonal_host(A, nv))
    x_ref = spla.spsolve(A.to_scipy().tocsc(), b)
    Ao = oracle.Csr.from_matrix(A)
    xo, ro = oracle.gmres_simple(Ao, oracle.Simple(Ao, nv), b, restart=30, precond=oracle.PRE_BLOCK_DIAGONAL,
                                 rtol=1e-10, max_it=20000)
    x = np.zeros(A.shape[0])
    rep = cf.gmres_preconditioned(A, b, M, x, cf.IterativeSolverConfig(0.0, 1e-10, 20000), restart=30)
    assert rep.termination == cf.Termination.CONVERGED
    assert abs(rep.iterations - ro.iterations) <= 0.10 * ro.iterations + 5, (rep.iterations, ro.iterations)
    err, err_o = np.linalg.norm(x - x_ref), np.linalg.norm(xo - x_ref)
    assert err <= max(10 * err_o, 1e-9 * np.linalg.norm(x_ref)), (err, err_o)


def test_chain_on_stokes(cuda):
    """LinearSolverChain on the 16 x 16 Stokes system: GMRES + SIMPLE is the
    first tier that exists here and converges; with a budget of 20 iterations
    every tier fails and the chain reports it."""
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.chain import LinearSolverChain
    A, b, nv = P.stokes_2d_mac(16)
    x_ref = spla.spsolve(A.to_scipy().tocsc(), b)
    chain = LinearSolverChain(cf.IterativeSolverConfig(0.0, 1e-10, 20000)).with_krylov_restart(30)
    x = chain.solve(A, b, nv)
    assert chain.trace[-1][0] == "GMRES+SIMPLE" and chain.trace[-1][1].startswith("converged")
    assert np.linalg.norm(x - x_ref) <= 1e-8 * np.linalg.norm(x_ref)
    # warm: from a perturbed solution, to an absolute residual (a relative one
    # would be relative to the guess's already small residual)
    nb = np.linalg.norm(b)
    warm = LinearSolverChain(cf.IterativeSolverConfig(1e-9 * nb, 0.0, 20000)).with_krylov_restart(30)
    guess = x_ref * (1.0 + 1e-3 * np.random.default_rng(0).standard_normal(x_ref.shape[0]))
    x = warm.solve_with_guess(A, b, nv, guess)
    assert np.linalg.norm(b - A.to_scipy() @ x) <= 1.5e-9 * nb
    tight = LinearSolverChain(cf.IterativeSolverConfig(0.0, 1e-10, 20)).with_krylov_restart(30)
    with pytest.raises(cf.SolveError, match="all solver tiers failed"):
        tight.solve(A, b, nv)
    assert [t for t, _ in tight.trace if not _.startswith("skipped")][-1] == "BiCGSTAB"
