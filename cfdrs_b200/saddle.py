"""Saddle-point preconditioners (``cfd_saddle_setup``, ``cfd_simple_*``,
``cfd_block_diagonal_*``, ``cfd_component_block_*``).

``SimplePreconditioner`` and ``BlockDiagonalPreconditioner`` of
``crates/cfd-math/src/linear_solver/block_preconditioner.rs``, which
``LinearSolverChain`` pairs with GMRES for saddle-point systems
(``chain.rs:216-238``, ``265-285``). The first ``n_velocity`` unknowns are
velocities, the rest pressures. SIMPLE: setup extracts diag(A)^-1, the
divergence rows D, the gradient block G and the diagonal Schur approximation
diag(C - D diag(A)^-1 G) from the matrix's current values; the apply is
u* = diag(A)^-1 f, p = S^-1 (g - D u*), u = u* - diag(A)^-1 G p. Block
diagonal: z = r / d, d the momentum diagonal and, per pressure row, the
absolute row sum over the pressure block.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .device import Context, device_matrix
from .krylov import SolveError


class _SaddleSplit:
    """A velocity/pressure split set on the device copy of ``matrix``."""

    def __init__(self, matrix, n_velocity: int, n_pressure: int | None = None, ctx: Context | None = None):
        n = matrix.shape[0]
        if n_pressure is None:
            n_pressure = n - n_velocity
        if n_velocity < 0 or n_pressure < 0 or n_velocity + n_pressure != n or matrix.shape[1] != n:
            raise SolveError(f"SIMPLE needs a square matrix of n_velocity + n_pressure rows "
                             f"({n_velocity} + {n_pressure} != {matrix.shape})")
        self.matrix = matrix
        self.n_velocity = int(n_velocity)
        self.n_pressure = int(n_pressure)
        self.dm = device_matrix(matrix, ctx)
        self.ctx = self.dm.ctx
        _lib.check(_lib.load().cfd_saddle_setup(self.dm.h, self.n_velocity))

    _apply_fn = ""

    def apply(self, r):
        """z = M^-1 r for a float64 CUDA tensor."""
        import torch
        if not (isinstance(r, torch.Tensor) and r.is_cuda and r.dtype == torch.float64):
            raise SolveError("apply takes a float64 CUDA tensor")
        r = r.contiguous()
        z = torch.empty_like(r)
        self.ctx.set_stream(torch.cuda.current_stream(r.device).cuda_stream)
        try:
            fn = getattr(_lib.load(), self._apply_fn)
            _lib.check(fn(self.dm.h, C.c_void_p(r.data_ptr()), C.c_void_p(z.data_ptr())))
        finally:
            self.ctx.set_stream(None)
        return z


class SimplePreconditioner(_SaddleSplit):
    """``SimplePreconditioner::new(matrix, n_velocity, n_pressure)``. Use it
    with :func:`cfdrs_b200.gmres_preconditioned` on the same matrix object."""
    _apply_fn = "cfd_simple_apply"


class BlockDiagonalPreconditioner(_SaddleSplit):
    """``BlockDiagonalPreconditioner::new(matrix, n_velocity, n_pressure)``.
    Use it with :func:`cfdrs_b200.gmres_preconditioned` on the same matrix
    object."""
    _apply_fn = "cfd_block_diagonal_apply"


class ComponentBlockPreconditioner(_SaddleSplit):
    """``ComponentBlockPreconditioner::new(matrix, n_velocity, n_pressure)``
    (``block_preconditioner.rs:609-976``): the velocity block split into three
    equal, uncoupled components (component-major order), each solved exactly
    after its zero diagonals are stabilized with ``pivot_tolerance``; the
    pressure Schur complement lumped by signed row sums. Setup raises
    :class:`cfdrs_b200.CfdError` where the reference's constructor returns
    ``Err`` (components that do not split into three equal blocks, entries
    coupling two components, a singular or oversized block). Use it with
    :func:`cfdrs_b200.gmres_preconditioned` on the same matrix object."""
    _apply_fn = "cfd_component_block_apply"

    def __init__(self, matrix, n_velocity: int, n_pressure: int | None = None, ctx: Context | None = None,
                 pivot_tolerance: float = 1e-12):
        n = matrix.shape[0]
        if n_pressure is None:
            n_pressure = n - n_velocity
        if n_velocity < 0 or n_pressure < 0 or n_velocity + n_pressure != n or matrix.shape[1] != n:
            raise SolveError(f"component blocks need a square matrix of n_velocity + n_pressure rows "
                             f"({n_velocity} + {n_pressure} != {matrix.shape})")
        self.matrix = matrix
        self.n_velocity = int(n_velocity)
        self.n_pressure = int(n_pressure)
        self.pivot_tolerance = float(pivot_tolerance)
        self.dm = device_matrix(matrix, ctx)
        self.ctx = self.dm.ctx
        _lib.check(_lib.load().cfd_component_block_setup(self.dm.h, self.n_velocity, self.pivot_tolerance))


def _csr_args(matrix):
    rp = np.ascontiguousarray(matrix.row_ptr, dtype=np.int64)
    col = np.ascontiguousarray(matrix.col, dtype=np.int32)
    val = np.ascontiguousarray(matrix.val, dtype=np.float64)
    return rp, col, val


def block_diagonal_host(matrix, n_velocity: int) -> np.ndarray:
    """The block-diagonal inverse on the host (``cfd_block_diagonal_host``)."""
    rp, col, val = _csr_args(matrix)
    inv = np.zeros(matrix.shape[0])
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    _lib.check(_lib.load().cfd_block_diagonal_host(matrix.shape[0], p(rp), p(col), p(val), int(n_velocity),
                                                   p(inv)))
    return inv


def simple_apply_host(matrix, n_velocity: int, b) -> np.ndarray:
    """The same setup and apply on the host (``cfd_simple_apply_host``)."""
    rp, col, val = _csr_args(matrix)
    bb = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(matrix.shape[0])
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    _lib.check(_lib.load().cfd_simple_apply_host(matrix.shape[0], p(rp), p(col), p(val), int(n_velocity), p(bb),
                                                 p(x)))
    return x


__all__ = ["SimplePreconditioner", "BlockDiagonalPreconditioner", "ComponentBlockPreconditioner", "simple_apply_host", "block_diagonal_host"]
