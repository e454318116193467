"""GMRES + ComponentBlock on the device (the first iterative tier of
LinearSolverChain::solve, chain.rs:193-217; block_preconditioner.rs:609-976):
the device apply against the oracle's (dense device inverse against the
oracle's LU: 1e-11 relative), the reference's own test, the refusals, value
updates, and GMRES against the oracle's GMRES with the same preconditioner
(iterations within 10 % + 5, error against the direct solution within 10x the
oracle's own or 1e-9 relative; FP32 inside FP64 refinement: 1e-8 relative)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

pytestmark = pytest.mark.gpu


def from_entries(entries, n):
    from cfdrs_b200.sparse import CsrMatrix
    r, c, v = zip(*entries)
    M = sp.coo_matrix((v, (r, c)), shape=(n, n)).tocsr()
    return CsrMatrix(M.indptr.astype(np.int64), M.indices.astype(np.int64), M.data, M.shape)


def device_apply(M, r):
    import torch
    return M.apply(torch.tensor(r, device="cuda")).cpu().numpy()


def test_reference_golden(cuda, golden):
    import cfdrs_b200 as cf
    g = golden["component_block"]
    A = from_entries(g["entries"], len(g["b"]))
    z = device_apply(cf.ComponentBlockPreconditioner(A, g["n_velocity"]), np.array(g["b"]))
    assert np.max(np.abs(z - np.array(g["x"]))) < g["tol"]


@pytest.mark.parametrize("n,eps", [(6, 0.1), (8, 0.0), (12, 0.1)])
def test_device_apply_matches_oracle(cuda, oracle, n, eps):
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    A, b, nv = P.stokes_3d_mac(n, eps=eps, seed=n)
    r = np.random.default_rng(n).standard_normal(A.shape[0])
    zo = oracle.ComponentBlock(oracle.Csr.from_matrix(A), nv).apply(r)
    z = device_apply(cf.ComponentBlockPreconditioner(A, nv), r)
    assert np.linalg.norm(z - zo) <= 1e-11 * np.linalg.norm(zo)


def test_refusals_and_rules(cuda):
    import cfdrs_b200 as cf
    from cfdrs_b200 import _lib
    from cfdrs_b200 import problems as P
    base = [[i, i, 4.0] for i in range(6)] + [[0, 6, -1.0], [6, 0, -1.0], [7, 7, 1.0]]
    A = from_entries(base, 8)
    with pytest.raises(_lib.CfdError) as e:
        cf.ComponentBlockPreconditioner(A, 4)
    assert e.value.status == 1
    with pytest.raises(_lib.CfdError, match="coupling") as e:
        cf.ComponentBlockPreconditioner(from_entries(base + [[0, 2, 0.5]], 8), 6)
    assert e.value.status == 2
    cf.ComponentBlockPreconditioner(from_entries(base + [[0, 2, 1e-15]], 8), 6)  # at most 1e-14: ignored
    singular = [[0, 0, 1.0], [0, 1, 1.0], [1, 0, 1.0], [1, 1, 1.0]] + [[i, i, 4.0] for i in range(2, 6)] + \
        [[6, 6, 1.0], [7, 7, 1.0]]
    with pytest.raises(_lib.CfdError, match="singular") as e:
        cf.ComponentBlockPreconditioner(from_entries(singular, 8), 6)
    assert e.value.status == 2
    # the 2-D MAC system: the velocity unknowns are two components, so a
    # three-way split couples neighbours across the cut and is refused
    A2, b2, nv2 = P.stokes_2d_mac(16)
    with pytest.raises(_lib.CfdError, match="coupling"):
        cf.ComponentBlockPreconditioner(A2, nv2)
    A3, b3, nv3 = P.stokes_3d_mac(6)
    M = cf.ComponentBlockPreconditioner(A3, nv3)
    cfg = cf.IterativeSolverConfig(0.0, 1e-10, 2000)
    with pytest.raises(cf.SolveError, match="GMRES"):
        cf.cg_preconditioned(A3, b3, M, np.zeros(A3.shape[0]), cfg)
    with pytest.raises(cf.SolveError, match="another matrix"):
        cf.gmres_preconditioned(A3.with_values(A3.val.copy()), b3, M, np.zeros(A3.shape[0]), cfg)


@pytest.mark.parametrize("n", [8, 12])
def test_gmres_component_block_matches_oracle(cuda, oracle, n):
    import torch
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    A, b, nv = P.stokes_3d_mac(n)
    x_ref = spla.spsolve(A.to_scipy().tocsc(), b)
    Ao = oracle.Csr.from_matrix(A)
    xo, ro = oracle.gmres_component_block(Ao, oracle.ComponentBlock(Ao, nv), b, restart=30, rtol=1e-10,
                                          max_it=5000)
    assert ro.termination == "Converged"
    M = cf.ComponentBlockPreconditioner(A, nv)
    cfg = cf.IterativeSolverConfig(0.0, 1e-10, 5000)
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


def test_value_updates_rebuild_the_blocks(cuda):
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.device import device_matrix
    A, b, nv = P.stokes_3d_mac(6)
    M = cf.ComponentBlockPreconditioner(A, nv)
    cfg = cf.IterativeSolverConfig(0.0, 1e-10, 2000)
    x1 = np.zeros(A.shape[0])
    assert cf.gmres_preconditioned(A, b, M, x1, cfg, restart=30).termination == cf.Termination.CONVERGED
    r = np.random.default_rng(2).standard_normal(A.shape[0])
    z1 = device_apply(M, r)
    device_matrix(A).update_values(2.0 * A.val)
    z2 = device_apply(M, r)  # rebuilt from the new values: (2A)'s preconditioner is half of A's
    assert np.linalg.norm(2.0 * z2 - z1) <= 1e-12 * np.linalg.norm(z1)
    x2 = np.zeros(A.shape[0])
    rep = cf.gmres_preconditioned(A, b, M, x2, cfg, restart=30)
    assert rep.termination == cf.Termination.CONVERGED
    assert np.linalg.norm(2.0 * x2 - x1) <= 1e-8 * np.linalg.norm(x1)


def test_chain_takes_the_component_tier(cuda):
    """LinearSolverChain::solve on the 8^3 Stokes system returns from GMRES +
    ComponentBlock; on the 2-D system that tier's setup is refused and GMRES +
    SIMPLE converges; the warm chain reaches the tier after SIMPLE."""
    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.chain import LinearSolverChain
    A, b, nv = P.stokes_3d_mac(8)
    x_ref = spla.spsolve(A.to_scipy().tocsc(), b)
    chain = LinearSolverChain(cf.IterativeSolverConfig(0.0, 1e-10, 5000)).with_krylov_restart(30)
    x = chain.solve(A, b, nv)
    assert chain.trace[-1][0] == "GMRES+ComponentBlock" and chain.trace[-1][1].startswith("converged")
    assert np.linalg.norm(x - x_ref) <= 1e-8 * np.linalg.norm(x_ref)
    A2, b2, nv2 = P.stokes_2d_mac(16)
    chain.solve(A2, b2, nv2)
    trace = dict(chain.trace)
    assert trace["GMRES+ComponentBlock"].startswith("setup failed") and trace["GMRES+SIMPLE"].startswith("converged")
