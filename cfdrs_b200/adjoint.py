"""Differentiable sparse solve: ``x = A^{-1} b`` as a ``torch.autograd.Function``
whose backward is hand-written on the device.

Backward of x = A^{-1} b for an upstream gradient g = dL/dx:
    lambda = A^{-T} g        (a second solve with the same preconditioner; A symmetric)
    dL/db  = lambda
    dL/dA  = -lambda x^T on A's sparsity pattern (cfd_pattern_outer)

Any differentiable assembly of A's values and b in torch (e.g.
:func:`darcy_2d_torch`, k = exp(theta) with harmonic-mean faces) then carries
the chain rule to its parameters. For the 2-D Darcy workload
:func:`darcy_2d_solve` does the assembly and the face-coefficient chain rule to
dL/dtheta each in one device kernel (``cfd_darcy2d_assemble``,
``cfd_darcy2d_theta_grad``), without a dL/dA array or an autograd graph
through the assembly. CFDrs has no differentiable solve; its Python
layer (``crates/cfd-python/src/lib.rs:85-158``) exposes physics solvers only, so
this module is new surface rather than a mirror.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .device import device_matrix, mark_synced
from .krylov import (IterativeSolverConfig, Precision, SolveError, SolveReport, Termination, bicgstab_preconditioned,
                     cg_preconditioned)
from .multigrid import AlgebraicMultigrid, AMGConfig, JacobiPreconditioner
from .sparse import CsrMatrix


class SparseSolver:
    """Device solver for a fixed sparsity pattern whose values come from torch.

    ``preconditioner``: "amg" (AMG-PCG; by default the pressure-Poisson
    configuration coarsened to at most 512 unknowns) or "jacobi". With AMG, :meth:`set_values`
    rebuilds the hierarchy when asked (``rebuild=True``) and otherwise follows
    ``refresh``: "recompute" re-forms the Galerkin operators for the new values
    with the cached transfer operators (``AlgebraicMultigrid::recompute``),
    "keep" leaves the hierarchy as it is (still an SPD preconditioner; only its
    quality for the new values changes, not the solution's accuracy).
    """

    def __init__(self, pattern: CsrMatrix, preconditioner: str = "amg", amg_config: AMGConfig | None = None,
                 precision: Precision = Precision.FP32_REFINE,
                 config: IterativeSolverConfig | None = None, solver: str = "cg"):
        self.pattern = CsrMatrix(pattern.row_ptr, pattern.col, pattern.val.copy(), pattern.shape)
        if self.pattern.nrows != self.pattern.ncols:
            raise SolveError("SparseSolver needs a square matrix")
        self.dm = device_matrix(self.pattern)
        if solver not in ("cg", "bicgstab"):
            raise SolveError(f"solver must be 'cg' or 'bicgstab', got {solver!r}")
        self.solver = solver
        self.kind = preconditioner
        if amg_config is None:
            # values change at every call, and with them (by the Galerkin
            # recompute) the coarsest operator's dense inverse, whose cost grows
            # with its size cubed: coarsen to at most 512 unknowns
            amg_config = AMGConfig.pressure_poisson()
            amg_config.min_coarse_size = 512
        self.amg_config = amg_config
        self.precision = precision
        self.config = config or IterativeSolverConfig(0.0, 1e-10, 2000)
        self.amg = None
        self.refresh = "recompute"
        # position of the transpose of every entry (symmetry check of the pattern)
        S = self.pattern.to_scipy().tocoo()
        key = S.row.astype(np.int64) * self.pattern.ncols + S.col
        keyT = S.col.astype(np.int64) * self.pattern.ncols + S.row
        order = np.argsort(key)
        pos = np.searchsorted(key[order], keyT)
        ok = (pos < key.size) & (key[order][np.minimum(pos, key.size - 1)] == keyT)
        self.pattern_symmetric = bool(ok.all())
        self._transpose_pos = order[np.minimum(pos, key.size - 1)] if self.pattern_symmetric else None
        self._transpose_dev = None
        self.symmetric = False

    def set_values(self, values: torch.Tensor, rebuild: bool = False) -> None:
        """New values (device float64, A's CSR order) for the fixed pattern.
        The device matrix and the library's host copy (read by AMG setup) take
        them; ``pattern`` keeps the values it was built with. Symmetry (for the
        adjoint) is checked on the device."""
        v = values.detach().to(dtype=torch.float64).contiguous()
        if v.numel() != self.pattern.nnz or not v.is_cuda:
            raise SolveError("values must be a CUDA float64 tensor with one entry per stored nonzero")
        self.dm.ctx.set_stream(torch.cuda.current_stream(v.device).cuda_stream)
        try:
            _lib.check(_lib.load().cfd_csr_set_values_device(self.dm.h, C.c_void_p(v.data_ptr())))
        finally:
            self.dm.ctx.set_stream(None)
        mark_synced(self.pattern, self.dm)
        if self.pattern_symmetric:
            if self._transpose_dev is None or self._transpose_dev.device != v.device:
                self._transpose_dev = torch.as_tensor(self._transpose_pos, device=v.device)
            self.symmetric = bool(torch.allclose(v, v[self._transpose_dev], rtol=1e-13, atol=0.0))
        else:
            self.symmetric = False
        if self.kind == "amg":
            if self.amg is None or rebuild:
                self.amg = AlgebraicMultigrid(self.dm, self.amg_config, ctx=self.dm.ctx)
            elif self.refresh == "recompute":
                self.amg.recompute(self.dm)

    def solve(self, b: torch.Tensor, precision: Precision | None = None,
              config: IterativeSolverConfig | None = None) -> torch.Tensor:
        x = torch.zeros_like(b, dtype=torch.float64)
        pre = self.amg if self.kind == "amg" else JacobiPreconditioner(self.dm)
        fn = cg_preconditioned if self.solver == "cg" else bicgstab_preconditioned
        rep = fn(self.dm, b.to(torch.float64).contiguous(), pre, x, config or self.config,
                 precision=self.precision if precision is None else precision)
        if rep.termination not in (Termination.CONVERGED, Termination.INITIAL_RESIDUAL):
            raise SolveError(f"sparse solve did not converge: {rep}")
        self.last_report = rep
        return x

    def adjoint(self, g: torch.Tensor, x: torch.Tensor, values: bool = True):
        """The backward of x = A^-1 b for g = dL/dx (``cfd_adjoint``): lambda =
        A^-T g, solved on A when A is symmetric (the forward's preconditioner)
        and on A's transpose otherwise (Jacobi preconditioner), and, with
        ``values``, dL/dA on A's pattern. Returns (lambda, dL/dA or None)."""
        g = g.to(torch.float64).contiguous()
        x = x.to(torch.float64).contiguous()
        lam = torch.empty_like(g)
        gv = torch.empty(self.pattern.nnz, dtype=torch.float64, device=g.device) if values else None
        transpose = not self.symmetric
        use_amg = self.kind == "amg" and not transpose
        opt = _lib.SolveOptionsC(0 if self.solver == "cg" else 1, 2 if use_amg else 1, int(self.precision), 1,
                                 1e-4, 20, 0, 30)
        cfg = self.config.to_c()
        rep = _lib.SolveReportC()
        self.dm.ctx.set_stream(torch.cuda.current_stream(g.device).cuda_stream)
        try:
            st = _lib.load().cfd_adjoint(self.dm.h, C.byref(opt), self.amg.h if use_amg else None,
                                         C.c_void_p(x.data_ptr()), C.c_void_p(g.data_ptr()),
                                         C.c_void_p(lam.data_ptr()), C.c_void_p(gv.data_ptr()) if values else None,
                                         1 if transpose else 0, C.byref(cfg), C.byref(rep))
        finally:
            self.dm.ctx.set_stream(None)
        if st != _lib.CFD_OK:
            raise SolveError(f"adjoint solve failed: {_lib.STATUS_NAMES.get(st, st)}: "
                             f"{_lib.load().cfd_last_error().decode()}")
        report = SolveReport(Termination(rep.termination), rep.iterations, rep.initial_residual,
                             rep.final_residual, rep.threshold, rep.outer_iterations, rep.device_ms)
        if report.termination not in (Termination.CONVERGED, Termination.INITIAL_RESIDUAL):
            raise SolveError(f"adjoint solve did not converge: {report}")
        self.last_report = report
        return lam, gv

    def pattern_outer(self, lam: torch.Tensor, x: torch.Tensor, scale: float = 1.0) -> torch.Tensor:
        """g_e = -scale * lam[row(e)] * x[col(e)] on A's pattern (device)."""
        g = torch.empty(self.pattern.nnz, dtype=torch.float64, device=lam.device)
        lam = lam.contiguous()
        x = x.contiguous()
        self.dm.ctx.set_stream(torch.cuda.current_stream(lam.device).cuda_stream)
        try:
            _lib.check(_lib.load().cfd_pattern_outer(self.dm.h, C.c_void_p(lam.data_ptr()),
                                                     C.c_void_p(x.data_ptr()), scale, C.c_void_p(g.data_ptr())))
        finally:
            self.dm.ctx.set_stream(None)
        return g


class SparseSolveFunction(torch.autograd.Function):
    """x = A(values)^{-1} b; gradients to ``values`` (on A's pattern) and ``b``."""

    @staticmethod
    def forward(ctx, values, b, solver: SparseSolver, rebuild: bool = False):
        solver.set_values(values, rebuild=rebuild)
        x = solver.solve(b)
        ctx.solver = solver
        ctx.save_for_backward(x)
        return x

    @staticmethod
    def backward(ctx, gx):
        solver: SparseSolver = ctx.solver
        (x,) = ctx.saved_tensors
        lam, gvals = solver.adjoint(gx, x)  # A^T lambda = dL/dx; dL/dA = -lambda x^T on the pattern
        return gvals, lam, None, None


def sparse_solve(values, b, solver: SparseSolver, rebuild: bool = False):
    return SparseSolveFunction.apply(values, b, solver, rebuild)


# ---------------------------------------------------------------------------
# 2-D Darcy assembly in torch (the same system as problems.darcy_2d).

def darcy_2d_pattern(n: int):
    """Pattern (CsrMatrix) and the (n, n, 5) mask of problems.darcy_2d."""
    from .problems import darcy_2d
    A, _ = darcy_2d(np.zeros((n, n)))
    mask = np.zeros((n, n, 5), dtype=bool)
    mask[1:, :, 0] = True
    mask[:, 1:, 1] = True
    mask[:, :, 2] = True
    mask[:, :-1, 3] = True
    mask[:-1, :, 4] = True
    return A, mask


def darcy_2d_torch(theta: torch.Tensor, mask: torch.Tensor):
    """CSR values and right-hand side of -div(exp(theta) grad p) = 0 on an n x n
    cell grid (row i + n*j), harmonic-mean faces, Dirichlet p = 1 (left) and
    p = 0 (right) at half a cell, no flux top/bottom; differentiable in theta."""
    n = theta.shape[0]
    k = torch.exp(theta)

    def hmean(a, b):
        return 2.0 * a * b / (a + b)

    fx = hmean(k[:, :-1], k[:, 1:])
    fy = hmean(k[:-1, :], k[1:, :])
    z = torch.zeros((n, n), dtype=theta.dtype, device=theta.device)
    south = torch.cat([torch.zeros((1, n), dtype=theta.dtype, device=theta.device), -fy], dim=0)
    north = torch.cat([-fy, torch.zeros((1, n), dtype=theta.dtype, device=theta.device)], dim=0)
    west = torch.cat([torch.zeros((n, 1), dtype=theta.dtype, device=theta.device), -fx], dim=1)
    east = torch.cat([-fx, torch.zeros((n, 1), dtype=theta.dtype, device=theta.device)], dim=1)
    wall = z.clone()
    wall = wall + torch.nn.functional.pad(2.0 * k[:, :1], (0, n - 1))
    wall = wall + torch.nn.functional.pad(2.0 * k[:, -1:], (n - 1, 0))
    diag = -(south + west + east + north) + wall
    vals = torch.stack([south, west, diag, east, north], dim=-1)
    values = vals[mask]
    b = torch.nn.functional.pad(2.0 * k[:, :1], (0, n - 1)).reshape(-1)
    return values, b


def darcy_2d_assemble_device(theta: torch.Tensor, solver: SparseSolver):
    """The values and right-hand side of :func:`darcy_2d_torch` from one
    kernel (``cfd_darcy2d_assemble``; the same operations, so the same bits),
    for the pattern of ``solver`` (:func:`darcy_2d_pattern`)."""
    n = theta.shape[0]
    th = theta.detach().to(torch.float64).contiguous()
    if not th.is_cuda or th.shape != (n, n):
        raise SolveError("theta must be an n x n CUDA tensor")
    vals = torch.empty(solver.pattern.nnz, dtype=torch.float64, device=th.device)
    b = torch.empty(n * n, dtype=torch.float64, device=th.device)
    solver.dm.ctx.set_stream(torch.cuda.current_stream(th.device).cuda_stream)
    try:
        _lib.check(_lib.load().cfd_darcy2d_assemble(solver.dm.h, n, C.c_void_p(th.data_ptr()),
                                                   C.c_void_p(vals.data_ptr()), C.c_void_p(b.data_ptr())))
    finally:
        solver.dm.ctx.set_stream(None)
    return vals, b


class DarcySolveFunction(torch.autograd.Function):
    """p = A(theta)^{-1} b(theta) for the 2-D Darcy system, with the assembly
    and the chain rule to theta each one kernel: forward assembles on the
    device and solves; backward solves the adjoint system with the same
    preconditioner and forms dL/dtheta in ``cfd_darcy2d_theta_grad`` (no dL/dA
    array, no autograd graph through the assembly)."""

    @staticmethod
    def forward(ctx, theta, solver: SparseSolver, rebuild: bool = False):
        vals, b = darcy_2d_assemble_device(theta, solver)
        solver.set_values(vals, rebuild=rebuild)
        x = solver.solve(b)
        ctx.solver = solver
        ctx.save_for_backward(theta.detach().to(torch.float64).contiguous(), x)
        return x

    @staticmethod
    def backward(ctx, gx):
        solver: SparseSolver = ctx.solver
        theta, x = ctx.saved_tensors
        lam, _ = solver.adjoint(gx, x, values=False)
        n = theta.shape[0]
        g = torch.empty_like(theta)
        solver.dm.ctx.set_stream(torch.cuda.current_stream(theta.device).cuda_stream)
        try:
            _lib.check(_lib.load().cfd_darcy2d_theta_grad(solver.dm.h, n, C.c_void_p(theta.data_ptr()),
                                                         C.c_void_p(lam.data_ptr()), C.c_void_p(x.data_ptr()),
                                                         C.c_void_p(g.data_ptr())))
        finally:
            solver.dm.ctx.set_stream(None)
        return g, None, None


def darcy_2d_solve(theta: torch.Tensor, solver: SparseSolver, rebuild: bool = False) -> torch.Tensor:
    """Differentiable p(theta) of the 2-D Darcy system (:class:`DarcySolveFunction`)."""
    return DarcySolveFunction.apply(theta, solver, rebuild)


def column_loss(p: torch.Tensor, n: int, column: int) -> torch.Tensor:
    """Sum of p^2 over the n cells of grid column ``column`` (row index i + n*j)."""
    return (p.reshape(n, n)[:, column] ** 2).sum()


def loss_column_index(n: int, x: float = 0.75) -> int:
    """First cell column whose centre (i + 1/2)/n is at or beyond ``x``."""
    return int(np.ceil(x * n - 0.5))
