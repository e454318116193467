"""Network assembly of the batched solver on the host (cfd_network_assemble_host:
the pattern step and the value code the device kernel runs), against the
oracle's restatement of MatrixAssembler::assemble_into
(crates/cfd-1d/src/solver/core/matrix_assembly.rs:163-250) bit for bit, and
the input checks of cfd_batch_create_networks."""
import ctypes as C

import numpy as np
import pytest

from cfdrs_b200 import _lib
from cfdrs_b200 import problems as P
from cfdrs_b200.batch import network_assemble_host, pack_networks


def oracle_batch(oracle, nets, neumann=None):
    """Per network through the oracle, concatenated as the batch lays it out."""
    rps, cols, vals, rhss = [0], [], [], []
    off = 0
    for s, n in enumerate(nets):
        q = None if neumann is None else neumann[off:off + n.n_nodes]
        A, b = oracle.network_assemble(n.n_nodes, n.edges_i, n.edges_j, n.conductance, n.fixed, n.fixed_value, q)
        rp, ci, v, _ = A.arrays()
        rps.extend((rp[1:] + rps[-1]).tolist())
        cols.append(ci)
        vals.append(v)
        rhss.append(b)
        off += n.n_nodes
    return np.array(rps), np.concatenate(cols), np.concatenate(vals), np.concatenate(rhss)


def tangled_network(rng, n, n_fixed, extra):
    """Parallel edges, both orientations, several fixed nodes (some joined to
    each other) and free nodes with several fixed neighbours."""
    ei = list(range(n - 1))
    ej = list(range(1, n))
    for _ in range(extra):
        a, c = (int(v) for v in rng.integers(0, n, size=2))
        if a != c:
            ei.append(a)
            ej.append(c)
    m = len(ei)
    fixed = np.zeros(n, np.int8)
    fixed[rng.choice(n, size=n_fixed, replace=False)] = 1
    return P.Network(n, np.array(ei, np.int32), np.array(ej, np.int32), rng.uniform(1e-3, 10.0, m), fixed,
                     rng.uniform(-50.0, 150.0, n) * fixed)


def same_bits(a, b):
    return a.shape == b.shape and np.array_equal(np.ascontiguousarray(a).view(np.int64),
                                                 np.ascontiguousarray(b).view(np.int64))


def check_against_oracle(oracle, nets, neumann=None):
    pk = pack_networks(nets)
    rp, col, val, rhs = network_assemble_host(pk, pk.conductance, neumann)
    orp, ocol, oval, orhs = oracle_batch(oracle, nets, neumann)
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
    assert same_bits(val, oval) and same_bits(rhs, orhs)
    return rp, col, val, rhs


def test_c4_networks_bit_for_bit(oracle):
    """The seeded C4-style networks (spanning tree + 10 % loops, node 0 and
    n - 1 fixed) at every size of the C4 range."""
    nets = P.network_batch_edges(48, seed=11, n_min=20, n_max=2000)
    check_against_oracle(oracle, nets)


@pytest.mark.parametrize("seed", range(6))
def test_tangled_networks_with_sources_bit_for_bit(oracle, seed):
    rng = np.random.default_rng(100 + seed)
    nets = [tangled_network(rng, int(rng.integers(2, 300)), int(rng.integers(0, 6)), int(rng.integers(0, 200)))
            for _ in range(int(rng.integers(1, 12)))]
    pk = pack_networks(nets)
    q = rng.standard_normal(pk.rows) if seed % 2 else None
    check_against_oracle(oracle, nets, q)


def test_reference_assembly_goldens(golden):
    """matrix_assembly.rs:270-450 through the product's host path."""
    for key, n, neumann in (("kirchhoff_abc", 3, None), ("kirchhoff_abc", 3, {1: 5.0}),
                            ("kirchhoff_active_block", 4, None)):
        g = golden[key]
        e = np.array(g["edges"])
        fixed, value = np.zeros(n, np.int8), np.zeros(n)
        for k, v in g["dirichlet"].items():
            fixed[int(k)], value[int(k)] = 1, v
        net = P.Network(n, e[:, 0].astype(np.int32), e[:, 1].astype(np.int32), e[:, 2], fixed, value)
        q = None
        if neumann:
            q = np.zeros(n)
            for k, v in neumann.items():
                q[k] = v
        rp, col, val, rhs = network_assemble_host(pack_networks([net]), net.conductance, q)
        import scipy.sparse as sp
        D = sp.csr_matrix((val, col, rp), shape=(n, n)).toarray()
        if key == "kirchhoff_abc":
            assert D[1, 1] == g["diag_b"] and D[0, 0] == 1.0 and D[2, 2] == 1.0
            assert rhs[1] == (g["rhs_b_with_neumann_5"] if neumann else g["rhs_b"])
            assert rhs[0] == 100.0 and rhs[2] == 0.0 and D[1, 0] == 0.0 and D[1, 2] == 0.0
        else:
            assert np.array_equal(D, np.array(g["dense"])) and np.array_equal(rhs, np.array(g["rhs"]))


def test_pattern_equals_problem_assembly():
    """The pattern the batch is built on equals problems.kirchhoff_assemble's
    (scipy), and the values agree up to the order of the diagonal sums."""
    nets = P.network_batch_edges(10, seed=4, n_min=20, n_max=900)
    pk = pack_networks(nets)
    rp, col, val, rhs = network_assemble_host(pk, pk.conductance)
    o = 0
    for net, (A, b) in zip(nets, P.network_batch(10, seed=4, n_min=20, n_max=900)):
        r0, r1 = o, o + net.n_nodes
        assert np.array_equal(rp[r0:r1 + 1] - rp[r0], A.row_ptr) and np.array_equal(col[rp[r0]:rp[r1]], A.col)
        np.testing.assert_allclose(val[rp[r0]:rp[r1]], A.val, rtol=64 * np.finfo(float).eps, atol=0)
        assert np.array_equal(rhs[r0:r1], b)
        o = r1


def _host_call(pk, g=None):
    L = _lib.load()
    nnz = C.c_int64()
    val = None if g is None else np.zeros(1 << 16)
    return L.cfd_network_assemble_host(pk.num_systems, _ptr(pk.node_off), _ptr(pk.edge_off), _ptr(pk.edge_i),
                                       _ptr(pk.edge_j), _ptr(pk.fixed), _ptr(pk.fixed_value), _ptr(g), None,
                                       C.byref(nnz), None, None, _ptr(val), None), L.cfd_last_error()


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _line(n=4):
    fixed = np.zeros(n, np.int8)
    fixed[0] = 1
    return P.Network(n, np.arange(n - 1, dtype=np.int32), np.arange(1, n, dtype=np.int32), np.ones(n - 1), fixed,
                     np.zeros(n))


@pytest.mark.parametrize("g,kind", [(np.nan, b"non-finite"), (np.inf, b"non-finite"), (-np.inf, b"non-finite"),
                                    (0.0, b"non-positive"), (-2.0, b"non-positive")])
def test_rejects_bad_conductance_naming_the_first_edge(g, kind):
    pk = pack_networks([_line(5), _line(4)])
    cond = np.ones(pk.edges)
    cond[5] = g
    cond[6] = -1.0
    st, msg = _host_call(pk, cond)
    assert st == 2 and kind in msg and b"at edge 5" in msg  # CFD_ERR_CONFIG


def test_rejects_malformed_networks():
    base = pack_networks([_line(4), _line(3)])

    def variant(**kw):
        d = dict(base.__dict__)
        d.update(kw)
        return type(base)(**d)
    ei = base.edge_i.copy()
    ei[4] = 2  # network 1's edge (1, 2) becomes the self-loop (2, 2)
    cases = [
        (variant(edge_i=ei), 2, b"self-loop edge 4"),
        (variant(edge_j=np.where(np.arange(base.edges) == 1, 9, base.edge_j).astype(np.int32)), 1,
         b"outside its 4 nodes"),
        (variant(node_off=np.array([0, 9, 7], np.int64)), 1, b"offsets decrease or pass"),
        (variant(edge_off=np.array([0, 6, 5], np.int64)), 1, b"offsets decrease or pass"),
        (variant(node_off=np.array([1, 4, 7], np.int64)), 1, b"must start at 0"),
        (variant(node_off=np.array([0, 4, -1], np.int64)), 1, b"must start at 0"),
    ]
    for pk, st_want, msg in cases:
        st, err = _host_call(pk)
        assert st == st_want and msg in err, (st, err)
    big = pack_networks([_line(2049)])
    st, err = _host_call(big)
    assert st == 1 and b"at most 2048" in err


def test_create_networks_checks_before_the_context():
    """cfd_batch_create_networks runs the same checks with no device, then
    reports the null context only for a valid description."""
    L = _lib.load()
    pk = pack_networks([_line(4), _line(3)])
    out = C.c_void_p(1)
    st = L.cfd_batch_create_networks(None, pk.num_systems, _ptr(pk.node_off), _ptr(pk.edge_off), _ptr(pk.edge_i),
                                     _ptr(pk.edge_j), _ptr(pk.fixed), _ptr(pk.fixed_value), C.byref(out))
    assert st == 7 and b"null context" in L.cfd_last_error() and not out.value
    bad = pack_networks([_line(2049)])
    st = L.cfd_batch_create_networks(None, bad.num_systems, _ptr(bad.node_off), _ptr(bad.edge_off),
                                     _ptr(bad.edge_i), _ptr(bad.edge_j), _ptr(bad.fixed), _ptr(bad.fixed_value),
                                     C.byref(out))
    assert st == 1 and b"at most 2048" in L.cfd_last_error()
    assert L.cfd_batch_assemble(None, None, None, 0) == 7


def test_degenerate_networks_bit_for_bit(oracle):
    """A single fixed node; a single free node without edges (an empty row);
    an edgeless network; every node fixed with edges only between fixed
    nodes (identity rows, nothing else); a free node isolated inside a
    network; parallel edges only."""
    N = P.Network
    i32 = lambda *v: np.array(v, np.int32)  # noqa: E731
    nets = [
        N(1, i32(), i32(), np.zeros(0), np.array([1], np.int8), np.array([7.5])),
        N(1, i32(), i32(), np.zeros(0), np.array([0], np.int8), np.zeros(1)),
        N(4, i32(), i32(), np.zeros(0), np.array([1, 0, 0, 1], np.int8), np.array([1.0, 0, 0, 2.0])),
        N(3, i32(0, 1, 0), i32(1, 2, 2), np.array([0.5, 0.25, 4.0]), np.ones(3, np.int8), np.array([1.0, 2.0, 3.0])),
        N(5, i32(0, 1, 3), i32(1, 3, 4), np.array([1.0, 2.0, 3.0]), np.array([1, 0, 0, 0, 1], np.int8),
          np.array([10.0, 0, 0, 0, -10.0])),
        N(2, i32(0, 1, 0, 1), i32(1, 0, 1, 0), np.array([1.0, 2.0, 3.0, 4.0]), np.array([0, 1], np.int8),
          np.array([0.0, 5.0])),
    ]
    rp, col, val, rhs = check_against_oracle(oracle, nets, np.linspace(-1, 1, sum(n.n_nodes for n in nets)))
    assert rp[2] - rp[1] == 0  # the lone free node: an empty row
    # network 4's node 2 (global 1 + 1 + 4 + 3 + 2 = 11) has no edge: empty row, RHS = its source
    assert rp[12] - rp[11] == 0
    # the all-fixed network: identity rows only
    k0, k1 = rp[6], rp[9]
    assert np.array_equal(val[k0:k1], np.ones(3)) and np.array_equal(col[k0:k1], [0, 1, 2])


def test_empty_batch():
    from cfdrs_b200.batch import PackedNetworks
    pk = PackedNetworks(np.zeros(1, np.int64), np.zeros(1, np.int64), np.zeros(0, np.int32), np.zeros(0, np.int32),
                        np.zeros(0, np.int8), np.zeros(0), np.zeros(0))
    rp, col, val, rhs = network_assemble_host(pk, pk.conductance)
    assert rp.tolist() == [0] and col.size == 0 and val.size == 0 and rhs.size == 0


def test_full_c4_workload_bit_for_bit(oracle):
    """All 4096 networks of the C4 workload (about 4.2 M nodes and 13 M
    entries), the full size the device assembly runs at."""
    nets = P.network_batch_edges(4096, seed=0)
    rp, col, val, rhs = check_against_oracle(oracle, nets)
    assert rp.shape[0] == sum(n.n_nodes for n in nets) + 1 and col.size > 13_000_000


def test_nonfinite_system_is_rejected():
    """validate_linear_system (solver_detection.rs:66-93): a fixed pressure or
    Neumann source that is not finite, or conductances whose sum overflows."""
    L = _lib.load()
    net = _line(4)
    pk = pack_networks([net])
    for kw, msg in ((dict(fixed_value=np.array([np.inf, 0, 0, 0])), b"RHS contains non-finite"),
                    (dict(conductance=np.array([1.7e308, 1.7e308, 1.0])), b"non-finite entry")):
        d = dict(pk.__dict__)
        d.update(kw)
        bad = type(pk)(**d)
        with pytest.raises(_lib.CfdError, match="non-finite") as e:
            network_assemble_host(bad, bad.conductance)
        assert e.value.status == 5 and msg in L.cfd_last_error()  # CFD_ERR_NONFINITE
    with pytest.raises(_lib.CfdError, match="RHS contains non-finite"):
        network_assemble_host(pk, pk.conductance, np.array([0.0, np.nan, 0.0, 0.0]))
