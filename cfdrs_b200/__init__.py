"""B200-native (sm_100a) sparse linear-solve path of CFDrs.

Drop-in for cfd-math's preconditioned Krylov surface: ``krylov`` (CG /
BiCGSTAB / GMRES entry points, reports and outcome mapping), ``multigrid`` (AMG
configuration and the device V-cycle), ``saddle`` (the SIMPLE and block-diagonal
saddle-point preconditioners), ``chain`` (``LinearSolverChain`` over them), ``pressure`` (the 2-D
pressure-correction dispatch), ``sparse`` (host CSR), ``problems``
(seeded assembly of the pressure / Kirchhoff systems). The compute runs in
``libcfdgpu.so`` through the C ABI of ``include/cfdgpu.h``.
"""
from .sparse import CsrMatrix, SparseMatrixBuilder, SparseError  # noqa: F401
from .krylov import (  # noqa: F401
    IterativeSolverConfig, Precision, SolveError, SolveOutcome, SolveReport, SolverKind, Termination,
    bicgstab, bicgstab_preconditioned, cg, cg_preconditioned, converged_or_none, gmres, gmres_preconditioned,
    gmres_width, interpret,
)
from .multigrid import (  # noqa: F401
    AMGConfig, AMGStatistics, AlgebraicMultigrid, CoarseOrder, CoarseSolve, CoarseningStrategy, HostHierarchy,
    IdentityPreconditioner, InterpolationStrategy, JacobiPreconditioner, SmootherType,
)
from .saddle import BlockDiagonalPreconditioner, ComponentBlockPreconditioner, SimplePreconditioner  # noqa: F401
from .chain import LinearSolverChain, LinearSolverState  # noqa: F401
from .pressure import PressureCorrectionDispatch, PressureLinearSolver  # noqa: F401

__version__ = "0.1.0"
