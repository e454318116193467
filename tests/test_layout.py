"""The SpMV device layout on the host: column codes, x windows, tails, index
records and code tables are walked with the kernels' own index arithmetic
(cfd_layout_check), every staged index is checked against its region and
against the column it must hold, and y = A x from that walk must equal the
CSR product."""
import numpy as np
import pytest
import scipy.sparse as sp

from cfdrs_b200 import problems as P
from cfdrs_b200.device import layout_check
from cfdrs_b200.sparse import CsrMatrix
from helpers import csr_from_lists, grid_laplacian


def random_csr(rng, n, ncols, lens):
    rp, col, val = [0], [], []
    for i in range(n):
        cols = np.sort(rng.choice(ncols, size=min(int(lens[i]), ncols), replace=False))
        col += cols.tolist()
        val += rng.uniform(-1, 1, cols.size).tolist()
        rp.append(len(col))
    return csr_from_lists(rp, col, val, ncols)


def check(A, seed=0):
    x = np.random.default_rng(seed).standard_normal(A.ncols)
    y, info = layout_check(A, x)
    ref = A.to_scipy() @ x
    np.testing.assert_allclose(y, ref, rtol=1e-14, atol=1e-14 * max(np.abs(ref).max(initial=0.0), 1.0))
    return info


@pytest.mark.parametrize("n", [5, 16, 33, 41])
def test_stencils_are_x_staged(n):
    """3-D 7-point operators, including sizes whose column count is not a
    multiple of 4 (the last window ends in a tail of 1-3 entries)."""
    info = check(P.poisson_3d_variable(n, 4.0, 1.0, seed=n)[0])
    assert info["all_compressed"] == 1 and info["x_staged"] == 1
    assert 1 <= info["max_windows"] <= 3


def test_2d_operators():
    assert check(grid_laplacian(37))["x_staged"] == 1
    A, _ = P.darcy_2d(P.gaussian_random_field((45, 45), 5.0, 0.5, seed=1))
    assert check(A)["x_staged"] == 1


def test_amg_levels(oracle):
    """Every operator of a modified-classical hierarchy (A, P, R per level), in
    both coarse numberings; each is checked whether or not it is x-staged."""
    A = P.poisson_3d_variable(24, 8.0, 1.0, seed=0)[0]
    staged = []
    for order in (0, 1):
        amg = oracle.Amg(oracle.Csr.from_matrix(A), oracle.AmgConfig(
            smoother=oracle.SMOOTH_JACOBI, relaxation=2 / 3, pre_smooth=1, post_smooth=1, interpolation=2,
            coarse_order=order, min_coarse_size=50, coarse_solve=oracle.COARSE_DENSE))
        for l in range(amg.num_levels):
            for which in ((0, 1, 2) if l < amg.num_levels - 1 else (0,)):
                rp, ci, v, shape = amg.level(l, which).arrays()
                staged.append(check(CsrMatrix(rp, ci, v, shape), seed=l)["x_staged"])
    assert staged[0] == 1 and sum(staged) >= 3


def test_ragged_rectangular_and_mixed():
    rng = np.random.default_rng(3)
    check(random_csr(rng, 3000, 3000, rng.integers(0, 12, 3000)))
    check(random_csr(rng, 700, 1900, rng.integers(0, 30, 700)))
    lens = rng.integers(1, 20, 600)
    lens[[5, 300, 599]] = [2500, 4096, 3001]
    info = check(random_csr(rng, 600, 5000, lens))  # rows beyond the staging capacity
    assert info["x_staged"] == 0
    S1 = P.poisson_3d_fv(12)[0].to_scipy()
    S2 = random_csr(rng, 1500, S1.shape[1], rng.integers(0, 40, 1500)).to_scipy()
    info = check(CsrMatrix.from_scipy(sp.vstack([S1, S2]).tocsr()))
    assert info["all_compressed"] == 0 and info["x_staged"] == 0


def test_empty_row_blocks():
    """A run of more than two blocks of empty rows between two stencils: the
    empty blocks stage only their row offsets and still produce y = 0."""
    S = P.poisson_3d_fv(10)[0].to_scipy()
    n = S.shape[0]
    A = CsrMatrix.from_scipy(sp.block_diag([S, sp.csr_matrix((1300, 1300)), S]).tocsr())
    info = check(A)
    assert info["x_staged"] == 1
    y, _ = layout_check(A, np.ones(A.ncols))
    assert np.all(y[n:n + 1300] == 0.0)


@pytest.mark.parametrize("ncols", [1, 2, 3, 5, 7])
def test_narrow_column_ranges(ncols):
    """Fewer than 4 columns (nothing to bulk-copy, the whole window is tail)
    and other column counts just past a 4-entry boundary."""
    rng = np.random.default_rng(ncols)
    A = random_csr(rng, 900, ncols, rng.integers(0, ncols + 1, 900))
    assert check(A)["x_staged"] == 1


def test_degenerate_shapes():
    check(csr_from_lists([0, 0, 0], [], [], 4))
    check(csr_from_lists([0, 1], [0], [2.0], 1))
    assert check(P.poisson_2d_dirichlet(64, seed=0)[0])["threads_per_row"] == 1


def test_networks():
    for A, _ in P.network_batch(4, seed=5, n_min=200, n_max=900):
        check(A)


def test_sliced_layout_on_stencils_and_levels(oracle):
    """The sliced layout (one warp per 32-row slice, slot-major values and
    codes) is built for one-thread rows with little padding and checked slot by
    slot against the CSR columns (cfd_layout_check runs check_sliced): the
    7-point and 5-point operators get it with under 1 % padding; every operator
    of a hierarchy is checked when it qualifies."""
    for A in (P.poisson_3d_variable(33, 4.0, 1.0, seed=2)[0], P.poisson_2d_dirichlet(70, seed=0)[0],
              grid_laplacian(41)):
        info = check(A)
        assert info["sliced"] == 1
        assert A.nnz <= info["sliced_slots"] <= 1.01 * A.nnz + 32 * 32
    A = P.poisson_3d_variable(24, 8.0, 1.0, seed=0)[0]
    amg = oracle.Amg(oracle.Csr.from_matrix(A), oracle.AmgConfig(
        smoother=oracle.SMOOTH_JACOBI, relaxation=2 / 3, pre_smooth=1, post_smooth=1, interpolation=2,
        coarse_order=1, min_coarse_size=50, coarse_solve=oracle.COARSE_DENSE))
    sliced = 0
    for l in range(amg.num_levels):
        for which in ((0, 1, 2) if l < amg.num_levels - 1 else (0,)):
            rp, ci, v, shape = amg.level(l, which).arrays()
            info = check(CsrMatrix(rp, ci, v, shape), seed=l)
            if info["sliced"]:
                sliced += 1
                assert info["sliced_slots"] <= 1.15 * len(ci) + 1
    assert sliced >= 1


def test_sliced_layout_refused_where_it_does_not_pay():
    rng = np.random.default_rng(9)
    # rows of 1 to 30 entries: padding far above 15 %
    assert check(random_csr(rng, 2000, 2000, rng.integers(1, 31, 2000)))["sliced"] == 0
    # a row longer than 32 entries
    lens = np.full(500, 5)
    lens[77] = 40
    assert check(random_csr(rng, 500, 500, lens))["sliced"] == 0
    # an empty matrix, and a single entry (one slice of 32 slots for one nonzero)
    assert check(csr_from_lists([0, 0, 0], [], [], 4))["sliced"] == 0
    assert check(csr_from_lists([0, 1], [0], [2.0], 1))["sliced"] == 0
    # a diagonal of 250 rows: the last slice is partial (rows past the end are padding)
    n = 250
    assert check(csr_from_lists(list(range(n + 1)), list(range(n)), [2.0] * n, n))["sliced"] == 1


def test_diagonal_layout_on_stencils():
    """Stencil operators get the diagonal layout (every entry on one of at most
    32 diagonals, at most 30 % empty slots); cfd_layout_check evaluates y = A x
    through it in the kernel's order and compares each row bit for bit with
    the CSR row sum of the other pipelines (check_diagonal), boundary rows with
    missing diagonals included."""
    # 5^3: the boundary rows leave 21 % of the slots empty, 3^3: 40 %
    cases = [(P.poisson_3d_variable(33, 4.0, 1.0, seed=2)[0], 7), (P.poisson_3d_variable(16, 4.0, 1.0, seed=3)[0], 7),
             (P.poisson_3d_variable(5, 4.0, 1.0, seed=3)[0], 7), (P.poisson_3d_variable(3, 4.0, 1.0, seed=3)[0], 0),
             (P.poisson_2d_dirichlet(70, seed=0)[0], 5), (grid_laplacian(41), 5),
             (csr_from_lists([0, 1], [0], [2.0], 1), 1)]
    for A, nd in cases:
        info = check(A)
        assert info["diagonals"] == nd, (A.shape, info["diagonals"])
    # a variable-coefficient 2-D Darcy operator
    A, _ = P.darcy_2d(P.gaussian_random_field((45, 45), 5.0, 0.5, seed=1))
    assert check(A)["diagonals"] == 5


def test_diagonal_layout_refused():
    rng = np.random.default_rng(4)
    n = 400
    # thirty-three distinct diagonals
    offs = list(range(-16, 17))
    rows = [[j for j in (i + o for o in offs) if 0 <= j < n] for i in range(n)]
    rp = np.concatenate([[0], np.cumsum([len(r) for r in rows])])
    A = csr_from_lists(rp.tolist(), sum(rows, []), rng.uniform(-1, 1, int(rp[-1])).tolist(), n)
    assert check(A)["diagonals"] == 0
    # eight diagonals, but far off-diagonal ones mostly outside the matrix: too many empty slots
    offs = [-300, -200, -1, 0, 1, 200, 300, 350]
    rows = [[j for j in (i + o for o in offs) if 0 <= j < n] for i in range(n)]
    rp = np.concatenate([[0], np.cumsum([len(r) for r in rows])])
    A = csr_from_lists(rp.tolist(), sum(rows, []), rng.uniform(-1, 1, int(rp[-1])).tolist(), n)
    assert check(A)["diagonals"] == 0
    # rectangular, empty, and one-thread-per-row violated (rows of 12 and more entries)
    assert check(random_csr(rng, 300, 200, np.full(300, 3)))["diagonals"] == 0
    assert check(csr_from_lists([0, 0, 0], [], [], 4))["diagonals"] == 0
    assert check(random_csr(rng, 300, 300, np.full(300, 30)))["diagonals"] == 0
    # an AMG Galerkin operator (irregular columns)
    assert check(P.network_batch(1, seed=5, n_min=200, n_max=300)[0][0])["diagonals"] == 0


def test_diagonal_layout_on_a_coarse_level():
    """The first coarse operator of the 64^3 Ruge-Stueben hierarchy (ascending
    coarse numbering) has 23 diagonals and two threads per row: the layout
    keeps per-row presence bits so its kernel adds every stored entry to the
    partial sum of its position, and check_diagonal compares that order with
    the CSR pipelines' bit for bit."""
    import cfdrs_b200 as cf
    from cfdrs_b200.multigrid import HostHierarchy
    A = P.poisson_3d_variable(64, 8.0, 1.0, seed=0)[0]
    H = HostHierarchy(A, cf.AMGConfig.pressure_poisson())
    info = check(H.level(1, 0))
    assert info["diagonals"] == 23 and info["threads_per_row"] == 2
    # the level below: hundreds of distinct offsets
    assert check(H.level(2, 0))["diagonals"] == 0
