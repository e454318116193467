"""ComponentBlockPreconditioner on the CPU (block_preconditioner.rs:609-976):
the oracle's restatement on the reference's own test, against an independent
numpy restatement on the 3-D MAC Stokes system, its refusals (split,
component coupling, singular block) and the oracle's GMRES + ComponentBlock
tier (chain.rs:193-217) against the direct solution."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from cfdrs_b200 import problems as P
from cfdrs_b200.sparse import CsrMatrix


def from_entries(entries, n):
    r, c, v = zip(*entries)
    M = sp.coo_matrix((v, (r, c)), shape=(n, n)).tocsr()
    return CsrMatrix(M.indptr.astype(np.int64), M.indices.astype(np.int64), M.data, M.shape)


def numpy_component_block(A, nv, b, pivot_tolerance=1e-12):
    """The same preconditioner restated with scipy/numpy: per component the
    stabilized block inverted densely, the Schur complement C - D diag(A)^-1 G
    (diag(A)^-1 = 1 where |a_ii| <= 1e-14) stabilized and lumped by signed row
    sums (the diagonal where the sum is at most 1e-14, 1 where both are)."""
    eps = 1e-14
    S = A.to_scipy().tocsr()
    n = S.shape[0]
    cs = nv // 3

    def stabilize(M):
        M = M.tolil()
        for r in range(M.shape[0]):
            row = M.getrow(r).toarray().ravel()
            scale = np.max(np.abs(row)) if row.size else 0.0
            if abs(row[r]) <= eps:
                M[r, r] = row[r] + max(scale * pivot_tolerance, eps)
        return M.tocsr()

    x = np.zeros(n)
    invs = []
    for c in range(3):
        blk = stabilize(S[c * cs:(c + 1) * cs, c * cs:(c + 1) * cs])
        invs.append(np.linalg.inv(blk.toarray()))
        x[c * cs:(c + 1) * cs] = invs[c] @ b[c * cs:(c + 1) * cs]
    d = S.diagonal()[:nv]
    dinv = np.where(np.abs(d) > eps, 1.0 / np.where(d == 0, 1, d), 1.0)
    G, D, Cb = S[:nv, nv:], S[nv:, :nv], S[nv:, nv:]
    schur = stabilize(Cb - D @ sp.diags(dinv) @ G)
    rs = np.asarray(schur.sum(axis=1)).ravel()
    sd = schur.diagonal()
    scale = np.where(np.abs(rs) > eps, rs, sd)
    pinv = np.where(np.abs(scale) > eps, 1.0 / np.where(scale == 0, 1, scale), 1.0)
    x[nv:] = (b[nv:] - D @ x[:nv]) * pinv
    gp = G @ x[nv:]
    for c in range(3):
        x[c * cs:(c + 1) * cs] -= invs[c] @ gp[c * cs:(c + 1) * cs]
    return x


def test_reference_golden(golden, oracle):
    """block_preconditioner.rs:1100-1116: u = (-2, -2, 0, 0, 0, 0), p = -12."""
    g = golden["component_block"]
    A = from_entries(g["entries"], len(g["b"]))
    x = oracle.ComponentBlock(oracle.Csr.from_matrix(A), g["n_velocity"]).apply(g["b"])
    assert np.max(np.abs(x - np.array(g["x"]))) < g["tol"]
    assert np.max(np.abs(numpy_component_block(A, g["n_velocity"], np.array(g["b"])) - g["x"])) < g["tol"]


@pytest.mark.parametrize("n,eps", [(4, 0.1), (6, 0.0), (8, 0.05)])
def test_oracle_equals_numpy_restatement(oracle, n, eps):
    """With and without a pressure block (eps = 0 leaves the Schur rows to
    the -D diag(A)^-1 G part alone)."""
    A, b, nv = P.stokes_3d_mac(n, eps=eps, seed=n)
    rng = np.random.default_rng(n)
    r = rng.standard_normal(A.shape[0])
    xo = oracle.ComponentBlock(oracle.Csr.from_matrix(A), nv).apply(r)
    xn = numpy_component_block(A, nv, r)
    assert np.linalg.norm(xo - xn) <= 1e-11 * np.linalg.norm(xn)


def test_zero_velocity_diagonal_is_stabilized(oracle):
    """A component row without a diagonal gets max(scale * 1e-12, 1e-14)."""
    A, b, nv = P.stokes_3d_mac(4, seed=3)
    S = A.to_scipy().tolil()
    S[0, 0] = 0.0
    M = sp.csr_matrix(S)
    M.eliminate_zeros()
    M.sort_indices()
    A0 = CsrMatrix(M.indptr.astype(np.int64), M.indices.astype(np.int64), M.data, M.shape)
    r = np.random.default_rng(1).standard_normal(A.shape[0])
    xo = oracle.ComponentBlock(oracle.Csr.from_matrix(A0), nv).apply(r)
    xn = numpy_component_block(A0, nv, r)
    assert np.linalg.norm(xo - xn) <= 1e-9 * np.linalg.norm(xn)


def test_refusals(oracle):
    """The constructor's Errs: a velocity count not divisible by three or
    beyond the system (1), an entry coupling two components (2), a block
    that stays singular after stabilization (3)."""
    g_entries = [[i, i, 4.0] for i in range(6)] + [[0, 6, -1.0], [6, 0, -1.0], [7, 7, 1.0]]
    A = oracle.Csr.from_matrix(from_entries(g_entries, 8))
    for bad in (4, 9):
        with pytest.raises(ValueError, match=r"\(1\)"):
            oracle.ComponentBlock(A, bad)
    coupled = oracle.Csr.from_matrix(from_entries(g_entries + [[0, 2, 0.5]], 8))
    with pytest.raises(ValueError, match=r"\(2\)"):
        oracle.ComponentBlock(coupled, 6)
    tiny = oracle.Csr.from_matrix(from_entries(g_entries + [[0, 2, 1e-15]], 8))
    oracle.ComponentBlock(tiny, 6)  # at most 1e-14: ignored
    singular = [[0, 0, 1.0], [0, 1, 1.0], [1, 0, 1.0], [1, 1, 1.0]] + [[i, i, 4.0] for i in range(2, 6)] + \
        [[6, 6, 1.0], [7, 7, 1.0]]
    with pytest.raises(ValueError, match=r"\(3\)"):
        oracle.ComponentBlock(oracle.Csr.from_matrix(from_entries(singular, 8)), 6)


def test_oracle_gmres_component_block_on_stokes(oracle):
    """GMRES(30) + ComponentBlock converges on the 8^3 Stokes system to the
    direct solution, in fewer iterations than GMRES + SIMPLE."""
    A, b, nv = P.stokes_3d_mac(8)
    x_ref = spla.spsolve(A.to_scipy().tocsc(), b)
    Ao = oracle.Csr.from_matrix(A)
    x, rep = oracle.gmres_component_block(Ao, oracle.ComponentBlock(Ao, nv), b, restart=30, rtol=1e-10,
                                          max_it=2000)
    assert rep.termination == "Converged"
    assert np.linalg.norm(x - x_ref) <= 1e-7 * np.linalg.norm(x_ref)
    _, rs = oracle.gmres_simple(Ao, oracle.Simple(Ao, nv), b, restart=30, rtol=1e-10, max_it=2000)
    assert rep.iterations < rs.iterations
