"""Saddle-point preconditioners on the CPU (SIMPLE and block diagonal): the
oracle's restatement (or_simple_*, or_block_diagonal_apply) on the
reference's own tests, the product's host path (cfd_simple_apply_host,
cfd_block_diagonal_host: the setup and the row code the device kernels run)
against the oracle bit for bit, edge cases of the velocity/pressure split,
and the oracle's GMRES with each on a MAC-grid Stokes system."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from cfdrs_b200 import _lib
from cfdrs_b200 import problems as P
from cfdrs_b200.saddle import simple_apply_host
from cfdrs_b200.sparse import CsrMatrix


def csr(M):
    M = sp.csr_matrix(M)
    M.sort_indices()
    return CsrMatrix(M.indptr.astype(np.int64), M.indices.astype(np.int64), M.data.astype(np.float64), M.shape)


def from_entries(entries, n):
    r, c, v = zip(*entries)
    # built from the listed entries only (a pressure row without a diagonal has none)
    M = sp.coo_matrix((v, (r, c)), shape=(n, n)).tocsr()
    return CsrMatrix(M.indptr.astype(np.int64), M.indices.astype(np.int64), M.data, M.shape)


def same_bits(a, b):
    return a.shape == b.shape and np.array_equal(np.ascontiguousarray(a).view(np.int64),
                                                 np.ascontiguousarray(b).view(np.int64))


@pytest.mark.parametrize("case", ["stabilized", "normalized"])
def test_reference_goldens(golden, oracle, case):
    """block_preconditioner.rs:1059-1085: the C - D diag(A)^-1 G = 3/4 system
    gives the exact solution; a normalized continuity row keeps its sign."""
    g = golden["simple_apply"]
    A = from_entries(g[case]["entries"], 4)
    want = np.array(g[case]["x"])
    xo = oracle.Simple(oracle.Csr.from_matrix(A), g["n_velocity"]).apply(g["b"])
    xp = simple_apply_host(A, g["n_velocity"], g["b"])
    assert np.max(np.abs(xo - want)) < g["tol"] and np.max(np.abs(xp - want)) < g["tol"]
    assert same_bits(xo, xp)


def random_saddle(rng, nv, np_, density=0.08, stab=True):
    """Momentum block with some zero or missing diagonals, a gradient block
    and a divergence block that is not its transpose (some D entries without
    a G partner), an optional pressure block."""
    A = sp.random(nv, nv, density=density, random_state=rng, data_rvs=lambda k: rng.uniform(-1, 1, k)).tolil()
    for i in range(nv):
        A[i, i] = rng.uniform(2, 5) if i % 7 else (0.0 if i % 14 else 1e-16)
    G = sp.random(nv, np_, density=density, random_state=rng, data_rvs=lambda k: rng.uniform(-1, 1, k))
    D = (G.T.tolil() * rng.uniform(0.5, 2.0)).tolil()
    extra = sp.random(np_, nv, density=density / 2, random_state=rng, data_rvs=lambda k: rng.uniform(-1, 1, k))
    D = (D + extra).tocsr()
    C = sp.diags(rng.uniform(-0.5, 0.5, np_)) if stab else sp.csr_matrix((np_, np_))
    return csr(sp.bmat([[A.tocsr(), G], [D, C]]))


@pytest.mark.parametrize("seed", range(8))
def test_host_path_equals_oracle_bit_for_bit(oracle, seed):
    rng = np.random.default_rng(seed)
    nv, np_ = int(rng.integers(5, 120)), int(rng.integers(1, 60))
    A = random_saddle(rng, nv, np_, stab=seed % 3 != 0)
    b = rng.standard_normal(nv + np_)
    xo = oracle.Simple(oracle.Csr.from_matrix(A), nv).apply(b)
    xp = simple_apply_host(A, nv, b)
    assert same_bits(xo, xp)


@pytest.mark.parametrize("n", [4, 9, 16, 64])
def test_stokes_host_path_equals_oracle(oracle, n):
    from cfdrs_b200.saddle import block_diagonal_host
    A, b, nv = P.stokes_2d_mac(n)
    S = oracle.Simple(oracle.Csr.from_matrix(A), nv)
    assert same_bits(S.apply(b), simple_apply_host(A, nv, b))
    assert same_bits(S.apply_block_diagonal(b), b * block_diagonal_host(A, nv))


def test_split_edge_cases(oracle):
    """All velocity (x = diag(A)^-1 b, identity where |a_ii| <= 1e-14), all
    pressure (x = diag^-1 b through the Schur diagonal), and a split outside
    [0, n]."""
    rng = np.random.default_rng(5)
    A = random_saddle(rng, 30, 10)
    b = rng.standard_normal(40)
    S = A.to_scipy()
    d = S.diagonal()
    inv = np.where(np.abs(d) > 1e-14, 1.0 / np.where(d == 0, 1, d), 1.0)
    assert same_bits(simple_apply_host(A, 40, b), b * inv)
    assert same_bits(simple_apply_host(A, 0, b), b * inv)
    for nv in (0, 40, 17):
        assert same_bits(simple_apply_host(A, nv, b), oracle.Simple(oracle.Csr.from_matrix(A), nv).apply(b))
    for bad in (-1, 41):
        with pytest.raises(_lib.CfdError, match="velocity unknowns outside"):
            simple_apply_host(A, bad, b)


def test_oracle_gmres_simple_on_stokes(oracle):
    """GMRES(30) + SIMPLE (chain.rs:216-238) on the 16 x 16 MAC Stokes system
    converges to the direct solution, in fewer iterations than unpreconditioned
    GMRES(30)."""
    A, b, nv = P.stokes_2d_mac(16)
    x_ref = spla.spsolve(A.to_scipy().tocsc(), b)
    Ao = oracle.Csr.from_matrix(A)
    x, rep = oracle.gmres_simple(Ao, oracle.Simple(Ao, nv), b, restart=30, rtol=1e-10, max_it=5000)
    assert rep.termination == "Converged"
    assert np.linalg.norm(x - x_ref) <= 1e-8 * np.linalg.norm(x_ref)
    _, rep_none = oracle.gmres(Ao, b, restart=30, rtol=1e-10, max_it=5000)
    assert rep.iterations < rep_none.iterations


def test_block_diagonal_golden(golden, oracle):
    """block_preconditioner.rs:1044-1058: u = 4/4, p = 1/1."""
    from cfdrs_b200.saddle import block_diagonal_host
    g = golden["simple_apply"]
    A = from_entries(g["stabilized"]["entries"], 4)
    bd = g["block_diagonal"]
    xo = oracle.Simple(oracle.Csr.from_matrix(A), g["n_velocity"]).apply_block_diagonal(bd["b"])
    xp = np.array(bd["b"]) * block_diagonal_host(A, g["n_velocity"])
    assert np.max(np.abs(xo - np.array(bd["x"]))) < g["tol"] and same_bits(xo, xp)


@pytest.mark.parametrize("seed", range(6))
def test_block_diagonal_host_equals_oracle(oracle, seed):
    """Including systems without a pressure block (every pressure row falls
    back to the mean |momentum diagonal|) and the all-velocity and
    all-pressure splits."""
    from cfdrs_b200.saddle import block_diagonal_host
    rng = np.random.default_rng(50 + seed)
    nv, np_ = int(rng.integers(5, 90)), int(rng.integers(1, 40))
    A = random_saddle(rng, nv, np_, stab=seed % 2 == 0)
    b = rng.standard_normal(nv + np_)
    for split in (nv, 0, nv + np_):
        xo = oracle.Simple(oracle.Csr.from_matrix(A), split).apply_block_diagonal(b)
        assert same_bits(xo, b * block_diagonal_host(A, split))


def test_oracle_gmres_block_diagonal_on_stokes(oracle):
    """GMRES(30) + block diagonal (chain.rs:265-285) converges on the 16 x 16
    Stokes system, between SIMPLE and no preconditioner in iterations."""
    A, b, nv = P.stokes_2d_mac(16)
    x_ref = spla.spsolve(A.to_scipy().tocsc(), b)
    Ao = oracle.Csr.from_matrix(A)
    S = oracle.Simple(Ao, nv)
    x, rep = oracle.gmres_simple(Ao, S, b, restart=30, precond=oracle.PRE_BLOCK_DIAGONAL, rtol=1e-10, max_it=5000)
    assert rep.termination == "Converged" and np.linalg.norm(x - x_ref) <= 1e-8 * np.linalg.norm(x_ref)
    _, rs = oracle.gmres_simple(Ao, S, b, restart=30, rtol=1e-10, max_it=5000)
    _, rn = oracle.gmres(Ao, b, restart=30, rtol=1e-10, max_it=5000)
    assert rs.iterations < rep.iterations < rn.iterations
