"""Batched network solve (cfd_batch_*) against the oracle's per-network
Jacobi-PCG with the row-equilibrated residual test.

Tolerances: every system must reach ||D(b - A x)|| <= 1e-10 ||D b|| when the
residual is recomputed on the host in FP64 (factor 1.5 allowed for the gap
between the recurrence and the true residual); iteration counts within 10 % (+5)
of the oracle's (CG on these kappa ~1e5 systems is sensitive to the order of
its reductions, so equal recurrences legitimately end a few percent apart);
the error against the direct solution no larger than 10x the oracle's own
error at the same tolerance (or 1e-9 relative); FP32 + refinement: error <= 1e-8
relative to the FP64 direct solution.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def eq_residual(A, x, b):
    S = A.to_scipy()
    s = 1.0 / np.abs(S).max(axis=1).toarray().ravel()
    return np.linalg.norm(s * (b - S @ x)) / np.linalg.norm(s * b)


@pytest.fixture(scope="module")
def batch(cuda):
    from cfdrs_b200 import problems as P
    from cfdrs_b200.batch import NetworkBatch
    from cfdrs_b200.sparse import CsrMatrix
    systems = P.network_batch(40, seed=5, n_min=20, n_max=700)
    # edge cases: a 1x1 system and a 2-node system with both nodes fixed
    systems.append((CsrMatrix([0, 1], [0], [2.0], (1, 1)), np.array([3.0])))
    systems.append(P.kirchhoff_assemble(2, [0], [1], [1e-12], {0: 5.0, 1: 1.0}))
    mats = [A for A, _ in systems]
    b = np.concatenate([b for _, b in systems])
    return NetworkBatch(mats), mats, b


def test_batch_fp64_matches_oracle(batch, oracle):
    import cfdrs_b200 as cf
    nb, mats, b = batch
    x, rep = nb.solve(b, config=cf.IterativeSolverConfig(0.0, 1e-10, 20000))
    assert rep.converged_systems == rep.num_systems == len(mats)
    import scipy.sparse.linalg as spla
    for A, xs, bs, it in zip(mats, nb.split(x), nb.split(b), rep.iterations):
        xo, ro = oracle.pcg_equilibrated(oracle.Csr.from_matrix(A), bs, rtol=1e-10)
        assert ro.termination in ("Converged", "InitialResidual")
        assert abs(int(it) - ro.iterations) <= 0.10 * ro.iterations + 5, (A.nrows, it, ro.iterations)
        assert eq_residual(A, xs, bs) <= 1.5e-10
        xd = spla.spsolve(A.to_scipy().tocsc(), bs)
        err_gpu = np.linalg.norm(xs - xd)
        err_oracle = np.linalg.norm(xo - xd)
        assert err_gpu <= max(10 * err_oracle, 1e-9 * np.linalg.norm(xd)), (A.nrows, err_gpu, err_oracle)


def test_batch_fp32_refinement(batch):
    import cfdrs_b200 as cf
    nb, mats, b = batch
    cfg = cf.IterativeSolverConfig(0.0, 1e-10, 40000)
    x64, r64 = nb.solve(b, config=cfg)
    x32, r32 = nb.solve(b, config=cfg, precision=cf.Precision.FP32_REFINE)
    assert r32.converged_systems == r32.num_systems
    import scipy.sparse.linalg as spla
    for A, xs, bs, xr in zip(mats, nb.split(x32), nb.split(b), nb.split(x64)):
        assert eq_residual(A, xs, bs) <= 1.5e-10
        xd = spla.spsolve(A.to_scipy().tocsc(), bs)
        # mixed precision: error <= 1e-8 against the FP64 direct solution
        assert np.linalg.norm(xs - xd) <= 1e-8 * np.linalg.norm(xd)


def test_batch_autotune_and_initial_guess(batch):
    import cfdrs_b200 as cf
    nb, mats, b = batch
    cfg = nb.autotune(cf.Precision.FP64, sample_iterations=32)
    assert all(t in (32, 64, 128, 256, 512) for t in cfg["threads"])
    assert all(g in (1, 2, 4) for g in cfg["systems_per_cta"])
    assert sum(cfg["systems"]) == len(mats)
    x, rep = nb.solve(b, config=cf.IterativeSolverConfig(0.0, 1e-10, 20000))
    assert rep.converged_systems == rep.num_systems
    # restarting from the solution: every system is already converged
    x2, rep2 = nb.solve(b, x=x, config=cf.IterativeSolverConfig(0.0, 1e-6, 20000))
    assert set(rep2.termination.tolist()) <= {int(cf.Termination.INITIAL_RESIDUAL), int(cf.Termination.CONVERGED)}


def test_batch_update_values(batch, oracle):
    import cfdrs_b200 as cf
    nb, mats, b = batch
    scaled = [A.with_values(A.val * (1.0 + 0.5 * (k % 3))) for k, A in enumerate(mats)]
    nb.update_values(np.concatenate([A.val for A in scaled]))
    x, rep = nb.solve(b, config=cf.IterativeSolverConfig(0.0, 1e-10, 20000))
    assert rep.converged_systems == rep.num_systems
    for A, xs, bs in zip(scaled, nb.split(x), nb.split(b)):
        assert eq_residual(A, xs, bs) <= 1.5e-10
    nb.update_values(np.concatenate([A.val for A in mats]))


def test_batch_rejects_oversized_system(cuda):
    from cfdrs_b200 import problems as P
    from cfdrs_b200.batch import NetworkBatch
    A, _ = P.poisson_2d_dirichlet(50)  # 2500 rows > 2048
    from cfdrs_b200 import _lib
    with pytest.raises(_lib.CfdError, match="at most"):
        NetworkBatch([A])


@pytest.mark.parametrize("precision", ["FP64", "FP32_REFINE"])
def test_batch_systems_per_cta_bit_identical(batch, precision):
    """Several systems per CTA (each on its own named barrier, or the warp
    barrier at 32 threads) give the results of one system per CTA at the same
    threads per system bit for bit."""
    import cfdrs_b200 as cf
    nb, mats, b = batch
    prec = cf.Precision[precision]
    cfg = cf.IterativeSolverConfig(0.0, 1e-10, 40000)
    saved = nb.config(prec)
    try:
        for thr in ([32, 32, 32, 32], [64, 64, 128, 128]):
            nb.set_config(thr, [1, 1, 1, 1], prec)
            x1, r1 = nb.solve(b, config=cfg, precision=prec)
            # the two large buckets' systems take more than half the shared
            # memory of an SM in FP64, so they stay at one per CTA
            for grp in ([2, 2, 1, 1], [4, 4, 1, 1], [2, 4, 2, 1]) if precision == "FP32_REFINE" else \
                    ([2, 2, 1, 1], [4, 4, 1, 1]):
                nb.set_config(thr, grp, prec)
                xg, rg = nb.solve(b, config=cfg, precision=prec)
                assert np.array_equal(x1.view(np.int64), xg.view(np.int64)), (thr, grp)
                assert np.array_equal(r1.iterations, rg.iterations)
                assert rg.converged_systems == rg.num_systems
    finally:
        nb.set_config(saved["threads"], saved["systems_per_cta"], prec)


def test_batch_set_config_rejects_bad_widths(batch):
    import cfdrs_b200 as cf
    from cfdrs_b200 import _lib
    nb, _, _ = batch
    with pytest.raises(_lib.CfdError):
        nb.set_config([48, 64, 64, 64], [1, 1, 1, 1])
    with pytest.raises(_lib.CfdError):
        nb.set_config([512, 64, 64, 64], [4, 1, 1, 1])
    with pytest.raises(_lib.CfdError):
        nb.set_config([64, 64, 64, 64], [3, 1, 1, 1])
