"""Shared test helpers: small matrices of the reference's unit tests."""
import numpy as np

from cfdrs_b200.sparse import CsrMatrix


def tridiag(n, lo=-1.0, d=2.0, hi=-1.0):
    rp, col, val = [0], [], []
    for i in range(n):
        if i > 0:
            col.append(i - 1); val.append(lo)
        col.append(i); val.append(d)
        if i < n - 1:
            col.append(i + 1); val.append(hi)
        rp.append(len(col))
    return CsrMatrix(rp, col, val, (n, n))


def grid_laplacian(n):
    """poisson_2d(n) of amg_integration_test.rs:17-48 (4 / -1, row-major)."""
    rp, col, val = [0], [], []
    for i in range(n * n):
        r, c = divmod(i, n)
        if r > 0:
            col.append(i - n); val.append(-1.0)
        if c > 0:
            col.append(i - 1); val.append(-1.0)
        col.append(i); val.append(4.0)
        if c + 1 < n:
            col.append(i + 1); val.append(-1.0)
        if r + 1 < n:
            col.append(i + n); val.append(-1.0)
        rp.append(len(col))
    return CsrMatrix(rp, col, val, (n * n, n * n))


def manufactured(size):
    t = np.arange(size) / size
    return np.sin(np.pi * t) + 0.5 * t


def csr_from_lists(rp, col, val, n=None):
    n = len(rp) - 1 if n is None else n
    return CsrMatrix(rp, col, val, (len(rp) - 1, n))
