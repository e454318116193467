"""Host CSR storage mirroring ``leto_ops::CsrMatrix`` as cfd-math uses it
(``crates/cfd-math/src/sparse/mod.rs:45-53``; fields ``values``,
``col_indices``, ``row_ptr`` as read at
``crates/cfd-math/src/linear_solver/preconditioners/multigrid/mod.rs:190-203``)
and the COO -> CSR ``SparseMatrixBuilder``
(``crates/cfd-math/src/sparse/builder.rs:71-330``).

Column indices are int32 and sorted within each row; row offsets are int64.
"""
from __future__ import annotations

import numpy as np


class SparseError(ValueError):
    """Structural error (maps to ``cfd_core::error::Error::InvalidConfiguration``)."""


class CsrMatrix:
    """CSR matrix. ``val`` is a read-only view: values change through
    :meth:`set_values`, which bumps :attr:`version` so that a device copy made
    earlier (``device.device_matrix``) is refreshed before its next use. The
    reference reads ``matrix.values()`` on every call, so a solve after a value
    change always sees the new values; a stale device copy would not."""

    __slots__ = ("row_ptr", "col", "_val", "shape", "version", "__weakref__")

    def __init__(self, row_ptr, col, val, shape):
        self.row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
        self.col = np.ascontiguousarray(col, dtype=np.int32)
        v = np.ascontiguousarray(val, dtype=np.float64).view()
        v.flags.writeable = False
        self._val = v
        self.version = 0
        self.shape = (int(shape[0]), int(shape[1]))
        if self.row_ptr.shape[0] != self.shape[0] + 1:
            raise SparseError("row_ptr length must be nrows + 1")
        if self.col.shape[0] != self._val.shape[0] or self.row_ptr[-1] != self.col.shape[0]:
            raise SparseError("col/val length must equal row_ptr[-1]")

    @property
    def val(self) -> np.ndarray:
        """The stored values (read-only view; see :meth:`set_values`)."""
        return self._val

    def set_values(self, values) -> None:
        """Replace the values (same pattern; the matrix keeps its own copy) and
        bump ``version`` (``values_mut()`` of the reference's CsrMatrix). The
        constructor keeps the caller's value array by reference, so values
        written into that array directly are not seen as a change."""
        v = np.ascontiguousarray(values, dtype=np.float64)
        if v.shape != self._val.shape:
            raise SparseError("value array must match the pattern's nnz")
        w = v.copy()
        w.flags.writeable = False
        self._val = w
        self.version += 1

    @classmethod
    def from_parts(cls, values, col_indices, row_ptr, nrows, ncols):
        """``CsrMatrix::from_parts(values, col_indices, row_ptr, nrows, ncols)``."""
        m = cls(row_ptr, col_indices, values, (nrows, ncols))
        if m.nnz and (m.col.min() < 0 or m.col.max() >= ncols):
            raise SparseError("column index out of range")
        if np.any(np.diff(m.row_ptr) < 0):
            raise SparseError("row_ptr must be non-decreasing")
        return m

    @classmethod
    def from_scipy(cls, m):
        m = m.tocsr()
        m.sort_indices()
        return cls(m.indptr, m.indices, m.data, m.shape)

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.col, self.row_ptr), shape=self.shape)

    @property
    def nrows(self) -> int:
        return self.shape[0]

    @property
    def ncols(self) -> int:
        return self.shape[1]

    @property
    def nnz(self) -> int:
        return int(self.col.shape[0])

    def diagonal(self) -> np.ndarray:
        rows = np.repeat(np.arange(self.nrows, dtype=np.int64), np.diff(self.row_ptr))
        d = np.zeros(self.nrows)
        hit = rows == self.col
        np.add.at(d, rows[hit], self.val[hit])
        return d

    def matvec(self, x: np.ndarray) -> np.ndarray:
        return self.to_scipy() @ x

    def with_values(self, values) -> "CsrMatrix":
        """Same sparsity pattern, new values (the ``recompute`` use case)."""
        v = np.ascontiguousarray(values, dtype=np.float64)
        if v.shape != self.val.shape:
            raise SparseError("value array must match the pattern's nnz")
        return CsrMatrix(self.row_ptr, self.col, v, self.shape)


class SparseMatrixBuilder:
    """COO accumulation with duplicate summation, then CSR (``builder.rs:71``)."""

    def __init__(self, nrows: int, ncols: int):
        self.nrows, self.ncols = int(nrows), int(ncols)
        self._r: list[int] = []
        self._c: list[int] = []
        self._v: list[float] = []

    def add_entry(self, row: int, col: int, value: float) -> None:
        if not (0 <= row < self.nrows and 0 <= col < self.ncols):
            raise SparseError(f"entry ({row}, {col}) outside {self.nrows}x{self.ncols}")
        self._r.append(row)
        self._c.append(col)
        self._v.append(float(value))

    def set_dirichlet_row(self, row: int, diag: float = 1.0) -> None:
        """Replace ``row`` by an identity row (``builder.rs:133``)."""
        keep = [k for k, r in enumerate(self._r) if r != row]
        self._r = [self._r[k] for k in keep]
        self._c = [self._c[k] for k in keep]
        self._v = [self._v[k] for k in keep]
        self.add_entry(row, row, diag)

    def build(self) -> CsrMatrix:
        import scipy.sparse as sp
        m = sp.coo_matrix((np.asarray(self._v, dtype=np.float64),
                           (np.asarray(self._r, dtype=np.int64), np.asarray(self._c, dtype=np.int64))),
                          shape=(self.nrows, self.ncols)).tocsr()
        m.sum_duplicates()
        m.sort_indices()
        return CsrMatrix(m.indptr, m.indices, m.data, m.shape)
