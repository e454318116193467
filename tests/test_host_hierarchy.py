"""AlgebraicMultigrid::new / setup / build_next_level (amg.rs:217-380) as the
product runs it before the upload, called through cfd_amg_setup_host (no GPU):
level by level equal to the oracle's restatement for every coarsening,
interpolation and coarse numbering, and holding the structural facts of the
reference's setup (R = P^T, Galerkin coarse operators, shrinking levels)."""
import ctypes as C
import itertools

import numpy as np
import pytest
import scipy.sparse as sp

from helpers import grid_laplacian


def matrices():
    from cfdrs_b200 import problems as P
    return {"variable_3d_12": P.poisson_3d_variable(12, 4.0, 1.0, seed=3)[0], "laplacian_2d_24": grid_laplacian(24)}


def host_config(coarsening, interp, order, **kw):
    import cfdrs_b200 as cf
    return cf.AMGConfig(max_levels=kw.get("max_levels", 16), min_coarse_size=kw.get("min_coarse_size", 60),
                        coarsening_strategy=cf.CoarseningStrategy(coarsening),
                        interpolation_strategy=cf.InterpolationStrategy(interp), coarse_order=cf.CoarseOrder(order))


@pytest.mark.parametrize("name", ["variable_3d_12", "laplacian_2d_24"])
@pytest.mark.parametrize("coarsening,interp,order", list(itertools.product((0, 1, 2), (0, 1, 2), (0, 1))))
def test_hierarchy_matches_oracle(oracle, name, coarsening, interp, order):
    """Ruge-Stueben (0), aggregation (1), PMIS (2) x classical (0), direct (1),
    modified classical (2) x selection (0) / ascending (1) coarse numbering:
    the same levels, patterns and values, bit for bit."""
    import cfdrs_b200 as cf
    A = matrices()[name]
    h = cf.HostHierarchy(A, host_config(coarsening, interp, order))
    o = oracle.Amg(oracle.Csr.from_matrix(A), oracle.AmgConfig(
        max_levels=16, min_coarse_size=60, coarsening=coarsening, interpolation=interp, coarse_order=order))
    assert h.num_levels == o.num_levels >= 2
    for level in range(h.num_levels):
        for which in (0, 1, 2):
            if which and level == h.num_levels - 1:
                continue
            mine = h.level(level, which)
            rp, ci, v, shape = o.level(level, which).arrays()
            assert mine.shape == shape, (level, which)
            np.testing.assert_array_equal(mine.row_ptr, rp)
            np.testing.assert_array_equal(mine.col, ci)
            np.testing.assert_array_equal(mine.val, v)


@pytest.mark.parametrize("interp", [0, 1, 2])
def test_hierarchy_structure(interp):
    """R_l = P_l^T exactly; A_{l+1} = (R_l A_l) P_l; levels shrink until the
    coarse-size or level limit; P_l maps coarse to fine; direct interpolation
    is piecewise constant (one unit weight per fine point)."""
    import cfdrs_b200 as cf
    A = matrices()["variable_3d_12"]
    h = cf.HostHierarchy(A, host_config(0, interp, 1))
    st = h.statistics()
    assert st.num_levels == h.num_levels >= 3
    assert st.level_sizes == sorted(st.level_sizes, reverse=True)
    assert st.level_sizes[-1] <= 60 or st.num_levels == 16
    assert st.operator_complexity == pytest.approx(sum(st.level_nnz) / st.level_nnz[0])
    for level in range(h.num_levels - 1):
        Al = h.level(level, 0).to_scipy()
        Pl = h.level(level, 1).to_scipy()
        Rl = h.level(level, 2).to_scipy()
        Ac = h.level(level + 1, 0).to_scipy()
        assert Pl.shape == (Al.shape[0], Ac.shape[0]) and Rl.shape == (Ac.shape[0], Al.shape[0])
        assert (Rl != Pl.T.tocsr()).nnz == 0
        galerkin = (Rl @ Al) @ Pl
        assert abs(galerkin - Ac).max() <= 1e-12 * abs(Ac).max()
        if interp == 1:  # piecewise constant: one unit weight per fine point, every coarse point used
            assert np.all(np.diff(Pl.indptr) == 1) and np.all(Pl.data == 1.0)
            assert np.unique(Pl.indices).size == Ac.shape[0]


def test_host_handle_limits():
    """A host-only hierarchy answers statistics and levels; anything that needs
    the device, a bad configuration and a bad matrix fail with a status."""
    import cfdrs_b200 as cf
    from cfdrs_b200 import _lib
    A = grid_laplacian(8)
    h = cf.HostHierarchy(A, cf.AMGConfig(min_coarse_size=10))
    L = _lib.load()
    assert L.cfd_amg_apply(h.h, C.c_void_p(8), C.c_void_p(8)) == 7  # CFD_ERR_STATE
    assert b"host only" in L.cfd_last_error()
    assert L.cfd_amg_set_path(h.h, 1, -1) == 7
    with pytest.raises(_lib.CfdError):
        cf.HostHierarchy(A, cf.AMGConfig(max_levels=0))
    with pytest.raises(_lib.CfdError):
        cf.HostHierarchy(sp.csr_matrix(np.ones((3, 4))))
    bad = A.to_scipy().tocsr()
    bad.indices[1], bad.indices[0] = bad.indices[0], bad.indices[1]  # unsorted row
    from cfdrs_b200.sparse import CsrMatrix
    with pytest.raises(_lib.CfdError):
        cf.HostHierarchy(CsrMatrix(bad.indptr.astype(np.int64), bad.indices.astype(np.int64), bad.data, bad.shape))
    cfg = _lib.AmgConfigC()
    L.cfd_amg_config_default(C.byref(cfg))
    out = C.c_void_p()
    assert L.cfd_amg_setup_host(-1, None, None, None, C.byref(cfg), C.byref(out)) == 1  # CFD_ERR_DIM
    assert not out.value


@pytest.mark.parametrize("points", [2, 3, 4])
@pytest.mark.parametrize("interp", [0, 2])
def test_truncated_interpolation_matches_oracle(oracle, interp, points):
    """max_interpolation_points (the argument interpolation.rs:42 accepts and
    the reference ignores): the product and the oracle truncate P identically,
    every row keeps at most k weights, and each truncated row keeps its sum."""
    import cfdrs_b200 as cf
    A = matrices()["variable_3d_12"]
    cfg = host_config(0, interp, 1)
    cfg.max_interpolation_points = points
    h = cf.HostHierarchy(A, cfg)
    o = oracle.Amg(oracle.Csr.from_matrix(A), oracle.AmgConfig(
        max_levels=16, min_coarse_size=60, coarsening=0, interpolation=interp, coarse_order=1,
        max_interp_points=points))
    full = cf.HostHierarchy(A, host_config(0, interp, 1))
    assert h.num_levels == o.num_levels
    for level in range(h.num_levels):
        for which in ((0, 1, 2) if level < h.num_levels - 1 else (0,)):
            mine = h.level(level, which)
            rp, ci, v, shape = o.level(level, which).arrays()
            np.testing.assert_array_equal(mine.row_ptr, rp)
            np.testing.assert_array_equal(mine.col, ci)
            np.testing.assert_array_equal(mine.val, v)
    P0, F0 = h.level(0, 1), full.level(0, 1)
    assert np.diff(P0.row_ptr).max() <= points
    S0, Sf = P0.to_scipy(), F0.to_scipy()
    np.testing.assert_allclose(np.asarray(S0.sum(axis=1)).ravel(), np.asarray(Sf.sum(axis=1)).ravel(),
                               rtol=1e-12, atol=1e-14)
    assert np.diff(F0.row_ptr).max() > points  # the full P had rows to cut
