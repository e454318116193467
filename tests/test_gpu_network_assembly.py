"""Device network assembly (cfd_batch_create_networks, cfd_batch_assemble)
against the host path of the same code (cfd_network_assemble_host, itself
equal to the oracle's assemble_into bit for bit on the CPU):

* values and right-hand sides bit for bit, host and device inputs, with and
  without Neumann sources;
* solves of the device-assembled batch bit for bit equal to solves of a batch
  built from the host-assembled matrices (so the FP32 copy the refined solve
  reads is equal too);
* a Picard-style loop (network_solver.rs:289-340): re-assemble from new
  conductances on the device and re-solve from the last iterate, checked
  against the host-assembled system;
* the state rules: no solve before an assembly, none after a rejected one, a
  solve's own b replaces the assembled one."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def same_bits(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.int64), b.view(np.int64))


@pytest.fixture(scope="module")
def nets():
    from cfdrs_b200 import problems as P
    nets = P.network_batch_edges(96, seed=21, n_min=20, n_max=2000)
    # a network whose two fixed nodes are also joined directly (that edge adds nothing)
    n = nets[0]
    nets.append(P.Network(n.n_nodes, np.append(n.edges_i, 0).astype(np.int32),
                          np.append(n.edges_j, n.n_nodes - 1).astype(np.int32), np.append(n.conductance, 1e-9),
                          n.fixed, n.fixed_value))
    return nets


def host_batch(pk, val, rhs):
    """A batch of the host-assembled matrices (cfd_batch_create)."""
    from cfdrs_b200.batch import NetworkBatch, network_assemble_host
    from cfdrs_b200.sparse import CsrMatrix
    rp, col, _, _ = network_assemble_host(pk)
    mats = []
    for s in range(pk.num_systems):
        r0, r1 = int(pk.node_off[s]), int(pk.node_off[s + 1])
        k0, k1 = int(rp[r0]), int(rp[r1])
        mats.append(CsrMatrix(rp[r0:r1 + 1] - k0, col[k0:k1].astype(np.int64), val[k0:k1], (r1 - r0, r1 - r0)))
    return NetworkBatch(mats), rhs


def test_device_assembly_bit_for_bit(cuda, nets):
    import torch
    from cfdrs_b200.batch import NetworkBatch, network_assemble_host
    nb = NetworkBatch.from_networks(nets)
    pk = nb.packed
    q = np.random.default_rng(1).standard_normal(pk.rows)
    for neumann in (None, q):
        nb.assemble(pk.conductance, neumann)
        val, rhs = nb.values()
        _, _, hv, hr = network_assemble_host(pk, pk.conductance, neumann)
        assert same_bits(val, hv) and same_bits(rhs, hr)
    g = pk.conductance * np.random.default_rng(2).uniform(0.5, 2.0, pk.edges)
    nb.assemble(torch.tensor(g, device="cuda"), torch.tensor(q, device="cuda"))
    val, rhs = nb.values()
    _, _, hv, hr = network_assemble_host(pk, g, q)
    assert same_bits(val, hv) and same_bits(rhs, hr)


def test_solves_equal_host_assembled_batch(cuda, nets):
    import cfdrs_b200 as cf
    from cfdrs_b200.batch import NetworkBatch, network_assemble_host
    nb = NetworkBatch.from_networks(nets)
    pk = nb.packed
    nb.assemble(pk.conductance)
    _, _, hv, hr = network_assemble_host(pk, pk.conductance)
    hb, b = host_batch(pk, hv, hr)
    cfg = cf.IterativeSolverConfig(0.0, 1e-10, 40000)
    for prec in (cf.Precision.FP64, cf.Precision.FP32_REFINE):
        xd, rd = nb.solve(None, config=cfg, precision=prec)
        xh, rh = hb.solve(b, config=cfg, precision=prec)
        assert rd.converged_systems == rd.num_systems == len(nets)
        assert same_bits(xd, xh)
        assert np.array_equal(rd.iterations, rh.iterations)


def test_picard_loop_on_device(cuda, nets):
    """Conductances change by a few percent per pass, as a flow-dependent
    resistance would change them; each pass re-assembles on the device and
    re-solves from the last iterate, on torch's stream, with no host copy of
    the matrix. Under an absolute tolerance the warm start needs fewer
    iterations than a cold one."""
    import torch
    import scipy.sparse as sp
    import cfdrs_b200 as cf
    from cfdrs_b200.batch import NetworkBatch, network_assemble_host
    nb = NetworkBatch.from_networks(nets)
    pk = nb.packed
    rng = np.random.default_rng(3)
    g = torch.tensor(pk.conductance, device="cuda")
    x = torch.zeros(pk.rows, dtype=torch.float64, device="cuda")
    cfg = cf.IterativeSolverConfig(1e-6, 0.0, 40000)
    nb.assemble(g)
    x, rep = nb.solve(None, x, config=cfg)
    assert rep.converged_systems == rep.num_systems
    for _ in range(3):
        g = g * torch.tensor(1.0 + 0.02 * rng.standard_normal(pk.edges), device="cuda").clamp(min=0.5)
        nb.assemble(g)
        x_prev = x.clone()
        x, warm = nb.solve(None, x, config=cfg)
        assert warm.converged_systems == warm.num_systems
        cold_x, cold = nb.solve(None, torch.zeros_like(x), config=cfg)
        assert warm.total_iterations < cold.total_iterations
        assert not torch.equal(x, x_prev)
    gh = g.cpu().numpy()
    rp, col, val, rhs = network_assemble_host(pk, gh)
    A = sp.csr_matrix((val, col.astype(np.int64) + np.repeat(
        np.repeat(pk.node_off[:-1], np.diff(pk.node_off)), np.diff(rp)), rp), shape=(pk.rows, pk.rows))
    xs = x.cpu().numpy()
    s = 1.0 / abs(A).max(axis=1).toarray().ravel()
    r = s * (rhs - A @ xs)
    for k in range(pk.num_systems):
        r0, r1 = int(pk.node_off[k]), int(pk.node_off[k + 1])
        assert np.linalg.norm(r[r0:r1]) <= 1.5e-6


def test_state_rules(cuda, nets):
    import cfdrs_b200 as cf
    from cfdrs_b200 import _lib
    from cfdrs_b200.batch import NetworkBatch
    from cfdrs_b200.krylov import SolveError
    nb = NetworkBatch.from_networks(nets[:5])
    pk = nb.packed
    cfg = cf.IterativeSolverConfig(0.0, 1e-10, 20000)
    with pytest.raises(SolveError, match="no assembled right-hand side"):
        nb.solve(None, config=cfg)
    with pytest.raises(SolveError, match="no valid matrix"):
        nb.solve(np.ones(pk.rows), config=cfg)
    nb.assemble(pk.conductance)
    x, rep = nb.solve(None, config=cfg)
    assert rep.converged_systems == rep.num_systems
    bad = pk.conductance.copy()
    bad[7], bad[9] = 0.0, np.nan
    with pytest.raises(_lib.CfdError, match="non-positive conductance 0 at edge 7"):
        nb.assemble(bad)
    with pytest.raises(SolveError, match="no assembled right-hand side"):
        nb.solve(None, config=cfg)
    with pytest.raises(SolveError, match="no valid matrix"):
        nb.solve(np.ones(pk.rows), config=cfg)
    nb.assemble(pk.conductance)
    x2, _ = nb.solve(None, config=cfg)
    assert same_bits(x, x2)
    _, rhs = nb.values()
    nb.solve(np.ones(pk.rows), config=cfg)  # replaces the assembled right-hand side
    with pytest.raises(SolveError, match="no assembled right-hand side"):
        nb.solve(None, config=cfg)
    nb.assemble(pk.conductance)
    nb.autotune(cf.Precision.FP64, sample_iterations=8)  # its b = 1 replaces it too
    with pytest.raises(SolveError, match="no assembled right-hand side"):
        nb.solve(None, config=cfg)
    x3, _ = nb.solve(rhs, config=cfg)  # the same system, b given by the caller
    # other CTA widths after the autotune: other reduction orders, so equal to
    # the solve tolerance, not bit for bit
    assert np.linalg.norm(x3 - x) <= 1e-8 * np.linalg.norm(x)


def test_nonfinite_system_rejected_on_device(cuda, nets):
    """A non-finite Neumann source makes a non-finite right-hand side, which
    the assembly rejects (validate_linear_system, solver_detection.rs:66-93);
    the batch then holds no matrix until a good assembly."""
    import cfdrs_b200 as cf
    from cfdrs_b200 import _lib
    from cfdrs_b200.batch import NetworkBatch
    from cfdrs_b200.krylov import SolveError
    nb = NetworkBatch.from_networks(nets[:3])
    pk = nb.packed
    q = np.zeros(pk.rows)
    q[5] = np.inf
    with pytest.raises(_lib.CfdError, match="RHS contains non-finite") as e:
        nb.assemble(pk.conductance, q)
    assert e.value.status == 5
    with pytest.raises(SolveError, match="no valid matrix"):
        nb.solve(np.ones(pk.rows), config=cf.IterativeSolverConfig(0.0, 1e-10, 20000))
    nb.assemble(pk.conductance)
    _, rep = nb.solve(None, config=cf.IterativeSolverConfig(0.0, 1e-10, 20000))
    assert rep.converged_systems == rep.num_systems


def test_entry_beyond_fp32_range_blocks_fp32_solves(cuda, nets):
    """A finite conductance above the FP32 range assembles (the FP64 values are
    exact) and the FP64 solve runs; the FP32 copy would be infinite, so an
    FP32 + refinement solve is refused until an assembly without such an entry."""
    import cfdrs_b200 as cf
    from cfdrs_b200.batch import NetworkBatch
    from cfdrs_b200.krylov import SolveError
    nb = NetworkBatch.from_networks(nets[:3])
    pk = nb.packed
    g = pk.conductance.copy()
    g[0] = 1e39  # finite in FP64, above FLT_MAX
    nb.assemble(g)
    cfg = cf.IterativeSolverConfig(0.0, 1e-10, 20000)
    _, rep = nb.solve(None, config=cfg)
    assert rep.num_systems == 3
    with pytest.raises(SolveError, match="FP32 range"):
        nb.solve(None, config=cfg, precision=cf.Precision.FP32_REFINE)
    nb.assemble(pk.conductance)
    _, rep = nb.solve(None, config=cfg, precision=cf.Precision.FP32_REFINE)
    assert rep.converged_systems == rep.num_systems
