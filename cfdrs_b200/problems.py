"""Seeded host-side CSR assembly for the pressure / Kirchhoff systems the
CFDrs callers hand to cfd-math's Krylov solvers.

Every generator returns a :class:`~cfdrs_b200.sparse.CsrMatrix` (int64 row
offsets, int32 column indices sorted within each row, float64 values) plus the
right-hand side. The matrices are scaled so their entries are O(1); relative
residuals are invariant under that scaling.

Reference semantics restated here:

* 2-D pressure Poisson (``poisson_2d_dirichlet``): the 5-point assembly of
  ``crates/cfd-2d/src/pressure_velocity/correction.rs:273-330`` -- off-diagonal
  ``-1/h^2`` toward each interior neighbour, and a Dirichlet wall adds ``1/h^2``
  to the diagonal (``:295-311``). Rows are ``x``-major,
  ``idx = (i-1)*(ny-2) + (j-1)`` (``:281``).
* 3-D / 2-D variable-coefficient finite-volume Poisson ``-div(k grad p) = f``:
  face coefficient is the harmonic mean ``2 k_P k_E / (k_P + k_E)``
  (``crates/cfd-2d/src/pressure_velocity/rhie_chow.rs:155``); a Dirichlet face
  at half a cell from the centre contributes ``2 k_P`` to the diagonal.
* Kirchhoff networks (``kirchhoff_network``): the grounded conductance
  Laplacian of ``crates/cfd-1d/src/solver/core/matrix_assembly.rs:163-250``
  (Dirichlet column elimination into the RHS, identity rows for fixed nodes),
  with Hagen-Poiseuille conductance ``g = pi d^4 / (128 mu L)``
  (``crates/cfd-1d/src/physics/resistance/models/bahrami_universal.rs:64``).
"""
from __future__ import annotations

from typing import NamedTuple

import numpy as np

from .sparse import CsrMatrix


def _uniform_rhs(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.uniform(-1.0, 1.0, size=n)


def _stencil_csr(n_rows: int, offsets: list[int], vals: np.ndarray, mask: np.ndarray) -> CsrMatrix:
    """Assemble CSR from per-row stencil columns ``row + offsets[q]`` (ascending)."""
    counts = mask.sum(axis=1, dtype=np.int64)
    row_ptr = np.zeros(n_rows + 1, dtype=np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    rows = np.arange(n_rows, dtype=np.int64)
    cols = np.empty(mask.shape, dtype=np.int32)
    for q, off in enumerate(offsets):
        cols[:, q] = (rows + off).astype(np.int32, copy=False) if n_rows < 2**31 else rows + off
    col = cols[mask]
    val = vals[mask]
    return CsrMatrix(row_ptr, col, val, (n_rows, n_rows))


def poisson_2d_dirichlet(nx: int, ny: int | None = None, seed: int = 0):
    """2-D pressure Poisson on an ``nx x ny`` cell grid, homogeneous Dirichlet on
    all four walls, scaled by ``h^2`` (diagonal 4, off-diagonals -1).

    Returns ``(A, b)`` with ``b ~ U[-1, 1]`` i.i.d. from ``seed``.
    """
    ny = nx if ny is None else ny
    n = nx * ny
    i = np.arange(n, dtype=np.int64) // ny  # x index
    j = np.arange(n, dtype=np.int64) % ny   # y index
    offsets = [-ny, -1, 0, 1, ny]
    mask = np.ones((n, 5), dtype=bool)
    vals = np.full((n, 5), -1.0)
    mask[:, 0] = i > 0
    mask[:, 1] = j > 0
    mask[:, 3] = j < ny - 1
    mask[:, 4] = i < nx - 1
    # Diagonal: interior neighbours plus 1 per Dirichlet wall (correction.rs:295-311)
    # gives 4 in every row on a uniform grid.
    vals[:, 2] = 4.0
    return _stencil_csr(n, offsets, vals, mask), _uniform_rhs(n, seed)


def poisson_3d_fv(n: int, k: np.ndarray | None = None, seed: int = 0,
                  dirichlet_x: bool = True):
    """Cell-centred 7-point finite-volume ``-div(k grad p) = f`` on an ``n^3``
    grid (row index ``i + n*j + n^2*l``, ``i`` along x), scaled by ``1/h``.

    Faces carry the harmonic mean of the two cell coefficients. Dirichlet
    (``p = 0``) on the x = 0 and x = 1 faces contributes ``2 k_P``; all other
    faces are Neumann (no flux). ``k=None`` means ``k = 1``.
    """
    N = n ** 3
    if k is None:
        kk = np.ones((n, n, n))
    else:
        kk = np.asarray(k, dtype=np.float64).reshape(n, n, n)  # [l, j, i]
    def hmean(a, b):
        return 2.0 * a * b / (a + b)
    # Face coefficients along each axis, stored on the lower cell.
    fx = hmean(kk[:, :, :-1], kk[:, :, 1:])   # (n, n, n-1) faces between i and i+1
    fy = hmean(kk[:, :-1, :], kk[:, 1:, :])
    fz = hmean(kk[:-1, :, :], kk[1:, :, :])
    offsets = [-n * n, -n, -1, 0, 1, n, n * n]
    vals = np.zeros((n, n, n, 7))
    mask = np.zeros((n, n, n, 7), dtype=bool)
    vals[1:, :, :, 0] = -fz
    mask[1:, :, :, 0] = True
    vals[:, 1:, :, 1] = -fy
    mask[:, 1:, :, 1] = True
    vals[:, :, 1:, 2] = -fx
    mask[:, :, 1:, 2] = True
    vals[:, :, :-1, 4] = -fx
    mask[:, :, :-1, 4] = True
    vals[:, :-1, :, 5] = -fy
    mask[:, :-1, :, 5] = True
    vals[:-1, :, :, 6] = -fz
    mask[:-1, :, :, 6] = True
    diag = -(vals[..., 0] + vals[..., 1] + vals[..., 2] + vals[..., 4] + vals[..., 5] + vals[..., 6])
    if dirichlet_x:
        diag[:, :, 0] += 2.0 * kk[:, :, 0]
        diag[:, :, -1] += 2.0 * kk[:, :, -1]
    vals[..., 3] = diag
    mask[..., 3] = True
    A = _stencil_csr(N, offsets, vals.reshape(N, 7), mask.reshape(N, 7))
    return A, _uniform_rhs(N, seed)


def gaussian_random_field(shape: tuple[int, ...], corr_len: float, sigma: float,
                          seed: int) -> np.ndarray:
    """Seeded stationary Gaussian random field with squared-exponential
    covariance ``sigma^2 exp(-r^2 / (2 corr_len^2))`` (lengths in cells), by
    spectral synthesis on the periodic box: white noise filtered by the square
    root of the spectral density ``exp(-|kappa|^2 corr_len^2 / 2)``, then
    normalised to zero mean and standard deviation ``sigma``.
    """
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(shape)
    W = np.fft.rfftn(w)
    k2 = np.zeros(W.shape)
    for ax, m in enumerate(shape):
        if ax == len(shape) - 1:
            f = np.fft.rfftfreq(m)
        else:
            f = np.fft.fftfreq(m)
        kap = 2.0 * np.pi * f
        sh = [1] * len(shape)
        sh[ax] = W.shape[ax]
        k2 = k2 + (kap ** 2).reshape(sh)
    W *= np.exp(-0.25 * k2 * corr_len ** 2)
    g = np.fft.irfftn(W, s=shape, axes=tuple(range(len(shape))))
    g -= g.mean()
    g *= sigma / g.std()
    return g


def poisson_3d_variable(n: int, corr_len: float = 8.0, sigma: float = 1.0, seed: int = 0):
    """3-D variable-coefficient Poisson with ``k = exp(g)``, ``g`` a seeded GRF.

    Returns ``(A, b, k)``.
    """
    g = gaussian_random_field((n, n, n), corr_len, sigma, seed + 1)
    k = np.exp(g)
    A, b = poisson_3d_fv(n, k, seed=seed)
    return A, b, k


def darcy_2d(theta: np.ndarray):
    """2-D ``-div(exp(theta) grad p) = 0`` on an ``n x n`` cell grid (row index
    ``i + n*j``, ``i`` along x): Dirichlet ``p = 1`` on the left wall and ``p = 0``
    on the right wall (half-cell faces, ``2 k_P``), no flux top and bottom.

    Returns ``(A, b)``; ``b`` carries the left-wall Dirichlet flux ``2 k_P * 1``.
    """
    n = theta.shape[0]
    kk = np.exp(np.asarray(theta, dtype=np.float64)).reshape(n, n)  # [j, i]
    N = n * n
    def hmean(a, b):
        return 2.0 * a * b / (a + b)
    fx = hmean(kk[:, :-1], kk[:, 1:])
    fy = hmean(kk[:-1, :], kk[1:, :])
    offsets = [-n, -1, 0, 1, n]
    vals = np.zeros((n, n, 5))
    mask = np.zeros((n, n, 5), dtype=bool)
    vals[1:, :, 0] = -fy
    mask[1:, :, 0] = True
    vals[:, 1:, 1] = -fx
    mask[:, 1:, 1] = True
    vals[:, :-1, 3] = -fx
    mask[:, :-1, 3] = True
    vals[:-1, :, 4] = -fy
    mask[:-1, :, 4] = True
    diag = -(vals[..., 0] + vals[..., 1] + vals[..., 3] + vals[..., 4])
    diag[:, 0] += 2.0 * kk[:, 0]
    diag[:, -1] += 2.0 * kk[:, -1]
    vals[..., 2] = diag
    mask[..., 2] = True
    b = np.zeros((n, n))
    b[:, 0] = 2.0 * kk[:, 0] * 1.0
    A = _stencil_csr(N, offsets, vals.reshape(N, 5), mask.reshape(N, 5))
    return A, b.reshape(N)


def kirchhoff_assemble(n_nodes: int, edges_i, edges_j, conductance, dirichlet: dict, neumann: dict | None = None):
    """Grounded conductance Laplacian, ``MatrixAssembler::assemble_into``
    (``crates/cfd-1d/src/solver/core/matrix_assembly.rs:163-250``): a free-free
    edge adds the symmetric 2x2 Laplacian block; an edge to a Dirichlet node
    adds to the free node's diagonal and moves ``g p_D`` to its RHS; Neumann
    sources add to the RHS; Dirichlet nodes get identity rows with RHS ``p_D``.

    Raises ``ValueError`` on self loops and non-finite or non-positive
    conductances (``:184-203``). Returns ``(A, b)``.
    """
    import scipy.sparse as sp
    ei = np.asarray(edges_i, dtype=np.int64)
    ej = np.asarray(edges_j, dtype=np.int64)
    g = np.asarray(conductance, dtype=np.float64)
    if np.any(ei == ej):
        raise ValueError("Self-loop edge detected in network assembly")
    if not np.all(np.isfinite(g)):
        raise ValueError("Non-finite conductance encountered in network assembly")
    if np.any(g <= 0):
        raise ValueError("Non-positive conductance encountered in network assembly")
    is_dir = np.zeros(n_nodes, dtype=bool)
    pval = np.zeros(n_nodes)
    for node, p in dirichlet.items():
        is_dir[int(node)] = True
        pval[int(node)] = p
    di, dj = is_dir[ei], is_dir[ej]
    ff = ~di & ~dj
    rows = [ei[ff], ej[ff], ei[ff], ej[ff], ej[di & ~dj], ei[~di & dj], np.flatnonzero(is_dir)]
    cols = [ei[ff], ej[ff], ej[ff], ei[ff], ej[di & ~dj], ei[~di & dj], np.flatnonzero(is_dir)]
    vals = [g[ff], g[ff], -g[ff], -g[ff], g[di & ~dj], g[~di & dj], np.ones(int(is_dir.sum()))]
    b = np.zeros(n_nodes)
    np.add.at(b, ej[di & ~dj], g[di & ~dj] * pval[ei[di & ~dj]])
    np.add.at(b, ei[~di & dj], g[~di & dj] * pval[ej[~di & dj]])
    for node, q in (neumann or {}).items():
        b[int(node)] += q
    b[is_dir] = pval[is_dir]
    m = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(n_nodes, n_nodes)).tocsr()
    m.sum_duplicates()
    m.sort_indices()
    return CsrMatrix(m.indptr, m.indices, m.data, m.shape), b


def hagen_poiseuille_conductance(d, length, mu=1.0e-3):
    """``g = pi d^4 / (128 mu L)``, the inverse of the Hagen-Poiseuille
    resistance ``R = 128 mu L / (pi d^4)`` (``bahrami_universal.rs:64``)."""
    return np.pi * np.asarray(d) ** 4 / (128.0 * mu * np.asarray(length))


class Network(NamedTuple):
    """A pipe network as edges: node pair, conductance, and the Dirichlet
    nodes as a 0/1 mask with their pressures (one entry per node)."""
    n_nodes: int
    edges_i: np.ndarray
    edges_j: np.ndarray
    conductance: np.ndarray
    fixed: np.ndarray
    fixed_value: np.ndarray

    def dirichlet(self) -> dict:
        return {int(k): float(self.fixed_value[k]) for k in np.flatnonzero(self.fixed)}

    def assemble(self, neumann: dict | None = None):
        return kirchhoff_assemble(self.n_nodes, self.edges_i, self.edges_j, self.conductance, self.dirichlet(),
                                  neumann)


def random_network(n_nodes: int, rng: np.random.Generator, loop_fraction: float = 0.1,
                   p_in: float = 1000.0, p_out: float = 0.0):
    """Seeded pipe network (:func:`random_network_edges`) assembled by
    :func:`kirchhoff_assemble`. Returns ``(A, b)``."""
    return random_network_edges(n_nodes, rng, loop_fraction, p_in, p_out).assemble()


def random_network_edges(n_nodes: int, rng: np.random.Generator, loop_fraction: float = 0.1,
                         p_in: float = 1000.0, p_out: float = 0.0) -> Network:
    """Seeded pipe network: a random spanning tree (node i attaches to a uniform
    j < i) plus ``floor(loop_fraction * n)`` extra distinct edges; diameters
    U[50, 500] um, lengths U[1, 20] mm, mu = 1e-3 Pa s; node 0 fixed at ``p_in``,
    node n-1 at ``p_out``."""
    n = int(n_nodes)
    child = np.arange(1, n, dtype=np.int64)
    parent = np.minimum((rng.random(n - 1) * child).astype(np.int64), child - 1)
    ei = parent.tolist()
    ej = child.tolist()
    seen = set(zip(np.minimum(ei, ej).tolist(), np.maximum(ei, ej).tolist()))
    extra = int(np.floor(loop_fraction * n))
    while extra > 0:
        a, c = (int(v) for v in rng.integers(0, n, size=2))
        if a == c:
            continue
        key = (min(a, c), max(a, c))
        if key in seen:
            continue
        seen.add(key)
        ei.append(key[0])
        ej.append(key[1])
        extra -= 1
    m = len(ei)
    d = rng.uniform(50e-6, 500e-6, size=m)
    length = rng.uniform(1e-3, 20e-3, size=m)
    g = hagen_poiseuille_conductance(d, length)
    fixed = np.zeros(n, dtype=np.int8)
    fixed_value = np.zeros(n)
    fixed[[0, n - 1]] = 1
    fixed_value[0], fixed_value[n - 1] = p_in, p_out
    return Network(n, np.asarray(ei, dtype=np.int32), np.asarray(ej, dtype=np.int32), g, fixed, fixed_value)


def network_batch(num: int, seed: int = 0, n_min: int = 20, n_max: int = 2000, loop_fraction: float = 0.1):
    """``num`` seeded networks with node counts uniform in [n_min, n_max]
    (:func:`random_network` each). Returns a list of ``(A, b)``."""
    return [net.assemble() for net in network_batch_edges(num, seed, n_min, n_max, loop_fraction)]


def network_batch_edges(num: int, seed: int = 0, n_min: int = 20, n_max: int = 2000,
                        loop_fraction: float = 0.1) -> list[Network]:
    """The networks of :func:`network_batch` (same seed, same networks) as edges."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(n_min, n_max + 1, size=num)
    return [random_network_edges(int(n), rng, loop_fraction) for n in sizes]


def stokes_2d_mac(n: int, nu: float = 1.0, eps: float = 0.1, seed: int = 0):
    """2-D Stokes on an ``n x n`` cell MAC (staggered) grid of the unit square,
    a saddle-point system for the SIMPLE-preconditioned GMRES tier
    (``crates/cfd-math/src/linear_solver/chain.rs:216-238``).

    Unknowns: u on the interior vertical faces ((n-1) n), v on the interior
    horizontal faces (n (n-1)), then p per cell (n^2). Momentum rows: the
    viscous 5-point Laplacian (no-slip walls: normal faces are zero, a
    tangential wall adds nu/h^2 through the mirrored ghost) and the pressure
    gradient (p_right - p_left)/h; continuity rows D = G^T; pressure block
    -eps I (stabilisation, which removes the constant-pressure null space).
    The matrix is scaled by h^2. Returns ``(A, b, n_velocity)``, b a seeded
    body force in U[-1, 1] with zero continuity right-hand side."""
    import scipy.sparse as sp
    h = 1.0 / n
    nu_n = (n - 1) * n
    nv = 2 * nu_n
    rows, cols, vals = [], [], []

    def add(r, c, v):
        rows.append(r)
        cols.append(c)
        vals.append(v)

    def uid(i, j):  # face x = i h, 1 <= i <= n-1; cell row j
        return (i - 1) * n + j

    def vid(i, j):  # face y = j h, 1 <= j <= n-1; cell column i
        return nu_n + i * (n - 1) + (j - 1)

    def pid(i, j):
        return nv + i * n + j
    c = nu / (h * h)
    for i in range(1, n):
        for j in range(n):
            r = uid(i, j)
            d = 4.0 * c
            for ii in (i - 1, i + 1):
                if 1 <= ii <= n - 1:
                    add(r, uid(ii, j), -c)
            for jj in (j - 1, j + 1):
                if 0 <= jj <= n - 1:
                    add(r, uid(i, jj), -c)
                else:
                    d += c
            add(r, r, d)
            add(r, pid(i, j), 1.0 / h)
            add(r, pid(i - 1, j), -1.0 / h)
    for i in range(n):
        for j in range(1, n):
            r = vid(i, j)
            d = 4.0 * c
            for jj in (j - 1, j + 1):
                if 1 <= jj <= n - 1:
                    add(r, vid(i, jj), -c)
            for ii in (i - 1, i + 1):
                if 0 <= ii <= n - 1:
                    add(r, vid(ii, j), -c)
                else:
                    d += c
            add(r, r, d)
            add(r, pid(i, j), 1.0 / h)
            add(r, pid(i, j - 1), -1.0 / h)
    top = sp.coo_matrix((vals, (rows, cols)), shape=(nv, nv + n * n)).tocsr()
    G = top[:, nv:]
    D = G.T.tocsr()
    C = -eps * sp.identity(n * n, format="csr")
    M = sp.bmat([[top[:, :nv], G], [D, C]], format="csr") * (h * h)
    M.sum_duplicates()
    M.sort_indices()
    rng = np.random.default_rng(seed)
    b = np.concatenate([rng.uniform(-1.0, 1.0, nv), np.zeros(n * n)])
    return CsrMatrix(M.indptr, M.indices, M.data, M.shape), b, nv


def stokes_3d_mac(n: int, nu: float = 1.0, eps: float = 0.1, seed: int = 0):
    """3-D Stokes on an ``n x n x n`` cell MAC grid of the unit cube: the
    component-major saddle system of the GMRES + ComponentBlock tier
    (``crates/cfd-math/src/linear_solver/chain.rs:193-217``), whose velocity
    block has no cross-component entries and three equal components.

    Unknowns: u on the interior x-faces ((n-1) n^2), then v on the interior
    y-faces and w on the interior z-faces (the same count each), then p per
    cell (n^3). Momentum rows: the viscous 7-point Laplacian (no-slip walls:
    normal faces are zero, a tangential wall adds nu/h^2 through the mirrored
    ghost) and the pressure gradient along the component's axis; continuity
    rows D = G^T; pressure block -eps I. Scaled by h^2. Returns
    ``(A, b, n_velocity)``, b a seeded body force in U[-1, 1] with zero
    continuity right-hand side."""
    import scipy.sparse as sp
    h = 1.0 / n
    ncomp = (n - 1) * n * n
    nv = 3 * ncomp
    c = nu / (h * h)
    cell = lambda i, j, k: i + n * (j + n * k)  # noqa: E731
    rows, cols, vals = [], [], []
    for comp in range(3):
        # face index along `comp` runs 1..n-1; the two other axes 0..n-1
        ext = [n, n, n]
        ext[comp] = n - 1

        def fid(f):  # f = (i, j, k) with f[comp] in [1, n-1]
            g = list(f)
            g[comp] -= 1
            return comp * ncomp + g[0] + ext[0] * (g[1] + ext[1] * g[2])
        for a in range(1, n):
            for b_ in range(n):
                for d_ in range(n):
                    f = [0, 0, 0]
                    f[comp] = a
                    others = [ax for ax in range(3) if ax != comp]
                    f[others[0]] = b_
                    f[others[1]] = d_
                    r = fid(f)
                    diag = 6.0 * c
                    for ax in range(3):
                        for s in (-1, 1):
                            g = list(f)
                            g[ax] += s
                            if ax == comp:
                                if 1 <= g[ax] <= n - 1:
                                    rows.append(r); cols.append(fid(g)); vals.append(-c)
                            elif 0 <= g[ax] <= n - 1:
                                rows.append(r); cols.append(fid(g)); vals.append(-c)
                            else:
                                diag += c
                    rows.append(r); cols.append(r); vals.append(diag)
                    hi = list(f)
                    lo = list(f)
                    lo[comp] -= 1
                    rows.append(r); cols.append(nv + cell(*hi)); vals.append(1.0 / h)
                    rows.append(r); cols.append(nv + cell(*lo)); vals.append(-1.0 / h)
    top = sp.coo_matrix((vals, (rows, cols)), shape=(nv, nv + n ** 3)).tocsr()
    G = top[:, nv:]
    D = G.T.tocsr()
    C = -eps * sp.identity(n ** 3, format="csr")
    M = sp.bmat([[top[:, :nv], G], [D, C]], format="csr") * (h * h)
    M.sum_duplicates()
    M.sort_indices()
    rng = np.random.default_rng(seed)
    rhs = np.concatenate([rng.uniform(-1.0, 1.0, nv), np.zeros(n ** 3)])
    return CsrMatrix(M.indptr, M.indices, M.data, M.shape), rhs, nv
