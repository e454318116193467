"""ctypes front end of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the oracle; the product package never
imports it. The algorithms and their reference citations are in oracle.h.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# CFD_ORACLE_LIB selects another build of the oracle (e.g. the sanitizer build).
_LIB_PATH = os.environ.get("CFD_ORACLE_LIB") or os.path.join(_HERE, "liboracle.so")

RUGE_STUEBEN, AGGREGATION, PMIS = 0, 1, 2
SMOOTH_JACOBI, SMOOTH_GS, SMOOTH_SGS = 0, 1, 2
COARSE_SWEEPS, COARSE_DENSE = 0, 1
PRE_NONE, PRE_JACOBI, PRE_AMG = 0, 1, 2
TERMINATIONS = ["Converged", "InitialResidual", "MaxIterations", "Breakdown", "NonPositiveCurvature"]


def build() -> str:
    """Compile liboracle.so with the committed Makefile (no-op when up to date,
    and when CFD_ORACLE_LIB names a build made elsewhere)."""
    if not os.environ.get("CFD_ORACLE_LIB"):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class _AmgConfig(C.Structure):
    _fields_ = [("max_levels", C.c_int32), ("coarsening", C.c_int32),
                ("min_coarse_size", C.c_int64), ("interpolation", C.c_int32),
                ("smoother", C.c_int32), ("pre_smooth", C.c_int32), ("post_smooth", C.c_int32),
                ("relaxation", C.c_double), ("strength_threshold", C.c_double),
                ("coarse_solve", C.c_int32), ("coarse_sweeps", C.c_int32),
                ("aggregate_size", C.c_int64), ("seed", C.c_uint64), ("coarse_order", C.c_int32),
                ("max_interp_points", C.c_int32)]


class _SolverConfig(C.Structure):
    _fields_ = [("tolerance", C.c_double), ("relative_tolerance", C.c_double),
                ("max_iterations", C.c_int64)]


class _Report(C.Structure):
    _fields_ = [("termination", C.c_int32), ("pad", C.c_int32), ("iterations", C.c_int64),
                ("initial_residual", C.c_double), ("final_residual", C.c_double),
                ("threshold", C.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P, I64, D = C.c_void_p, C.c_int64, C.c_double
        L.or_csr_new.restype = P
        L.or_csr_new.argtypes = [I64, I64, I64, P, P, P]
        L.or_csr_info.argtypes = [P, P, P, P]
        L.or_csr_export.argtypes = [P, P, P, P]
        L.or_csr_free.argtypes = [P]
        L.or_set_threads.argtypes = [C.c_int]
        L.or_get_threads.restype = C.c_int
        L.or_spmv.argtypes = [P, P, P]
        L.or_strength.restype = P
        L.or_strength.argtypes = [P, D]
        L.or_transpose.restype = P
        L.or_transpose.argtypes = [P]
        L.or_spgemm.restype = P
        L.or_spgemm.argtypes = [P, P]
        L.or_coarsen.restype = I64
        L.or_coarsen.argtypes = [P, C.c_int, D, I64, C.c_uint64, C.c_int, P, P]
        L.or_classical_interp.restype = P
        L.or_classical_interp.argtypes = [P, P, I64, P]
        L.or_direct_interp.restype = P
        L.or_direct_interp.argtypes = [P, I64, I64]
        L.or_smooth.argtypes = [P, P, P, C.c_int, D, C.c_int]
        L.or_dense_solve.restype = C.c_int
        L.or_dense_solve.argtypes = [P, P, P]
        L.or_amg_setup.restype = P
        L.or_amg_setup.argtypes = [P, P]
        L.or_amg_from_levels.restype = P
        L.or_amg_from_levels.argtypes = [C.c_int, P, P, P, P]
        L.or_amg_num_levels.restype = C.c_int
        L.or_amg_num_levels.argtypes = [P]
        L.or_amg_level.restype = P
        L.or_amg_level.argtypes = [P, C.c_int, C.c_int]
        L.or_amg_apply.argtypes = [P, P, P]
        L.or_amg_free.argtypes = [P]
        L.or_pcg_equilibrated.restype = C.c_int
        L.or_pcg_equilibrated.argtypes = [P, P, P, P, P]
        for fn in (L.or_pcg, L.or_bicgstab):
            fn.restype = C.c_int
            fn.argtypes = [P, C.c_int, P, P, P, P, P, P]
        L.or_gmres.restype = C.c_int
        L.or_gmres.argtypes = [P, C.c_int, P, C.c_int64, P, P, P, P, P]
        L.or_gmres_width.restype = C.c_int
        L.or_gmres_width.argtypes = [C.c_int64]
        L.or_simple_new.restype = P
        L.or_simple_new.argtypes = [P, I64]
        L.or_simple_apply.argtypes = [P, P, P]
        L.or_simple_free.argtypes = [P]
        L.or_block_diagonal_apply.argtypes = [P, P, P]
        L.or_gmres_saddle.restype = C.c_int
        L.or_gmres_saddle.argtypes = [P, P, C.c_int, C.c_int64, P, P, P, P, P]
        L.or_detect_solver_method.restype = C.c_int
        L.or_detect_solver_method.argtypes = [P]
        L.or_dense_lu_solve.restype = C.c_int
        L.or_dense_lu_solve.argtypes = [I64, P, P]
        L.or_linear_system_solve.restype = C.c_int
        L.or_linear_system_solve.argtypes = [P, P, P, C.c_int, D, I64, P]
        L.or_component_block_new.restype = P
        L.or_component_block_new.argtypes = [P, I64, D, P]
        L.or_component_block_apply.argtypes = [P, P, P]
        L.or_component_block_free.argtypes = [P]
        L.or_gmres_component_block.restype = C.c_int
        L.or_gmres_component_block.argtypes = [P, P, I64, P, P, P, P, P]
        L.or_network_assemble.restype = C.c_int
        L.or_network_assemble.argtypes = [I64, I64, P, P, P, P, P, P, P, P, P]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class Csr:
    """Owned oracle CSR (int64 indices, float64 values)."""

    def __init__(self, handle, owned=True):
        self.h = handle
        self.owned = owned

    @classmethod
    def from_arrays(cls, row_ptr, col, val, shape):
        rp = np.ascontiguousarray(row_ptr, dtype=np.int64)
        ci = np.ascontiguousarray(col, dtype=np.int64)
        v = np.ascontiguousarray(val, dtype=np.float64)
        return cls(lib().or_csr_new(shape[0], shape[1], ci.shape[0], _ptr(rp), _ptr(ci), _ptr(v)))

    @classmethod
    def from_matrix(cls, m):
        """From any object with row_ptr/col/val/shape (e.g. cfdrs_b200.sparse.CsrMatrix)."""
        return cls.from_arrays(m.row_ptr, m.col, m.val, m.shape)

    def info(self):
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        lib().or_csr_info(self.h, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def arrays(self):
        nr, nc, nnz = self.info()
        rp = np.empty(nr + 1, np.int64)
        ci = np.empty(nnz, np.int64)
        v = np.empty(nnz, np.float64)
        lib().or_csr_export(self.h, _ptr(rp), _ptr(ci), _ptr(v))
        return rp, ci, v, (nr, nc)

    def to_scipy(self):
        import scipy.sparse as sp
        rp, ci, v, shape = self.arrays()
        return sp.csr_matrix((v, ci, rp), shape=shape)

    def spmv(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.info()[0])
        lib().or_spmv(self.h, _ptr(x), _ptr(y))
        return y

    def __del__(self):
        if getattr(self, "owned", False) and self.h:
            lib().or_csr_free(self.h)
            self.h = None


def strength(a: Csr, theta: float) -> Csr:
    return Csr(lib().or_strength(a.h, theta))


def transpose(a: Csr) -> Csr:
    return Csr(lib().or_transpose(a.h))


def spgemm(a: Csr, b: Csr) -> Csr:
    return Csr(lib().or_spgemm(a.h, b.h))


def coarsen(a: Csr, kind=RUGE_STUEBEN, theta=0.25, param=8, seed=0, literal_scan=False):
    n = a.info()[0]
    cp = np.empty(n, np.int64)
    f2c = np.empty(n, np.int64)
    nc = lib().or_coarsen(a.h, kind, theta, param, seed, int(literal_scan), _ptr(cp), _ptr(f2c))
    return cp[:nc].copy(), f2c


def classical_interp(a: Csr, coarse_points, s: Csr) -> Csr:
    cp = np.ascontiguousarray(coarse_points, dtype=np.int64)
    return Csr(lib().or_classical_interp(a.h, _ptr(cp), cp.shape[0], s.h))


def direct_interp(f2c, nc) -> Csr:
    m = np.ascontiguousarray(f2c, dtype=np.int64)
    return Csr(lib().or_direct_interp(_ptr(m), m.shape[0], nc))


def smooth(a: Csr, x, b, kind=SMOOTH_JACOBI, omega=1.0, iters=1):
    x = np.array(x, dtype=np.float64, copy=True)
    b = np.ascontiguousarray(b, dtype=np.float64)
    lib().or_smooth(a.h, _ptr(x), _ptr(b), kind, omega, iters)
    return x


def dense_solve(a: Csr, b):
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros_like(b)
    rc = lib().or_dense_solve(a.h, _ptr(b), _ptr(x))
    if rc != 0:
        raise ZeroDivisionError("singular coarse matrix")
    return x


@dataclass
class AmgConfig:
    max_levels: int = 10
    coarsening: int = RUGE_STUEBEN
    min_coarse_size: int = 50
    interpolation: int = 0  # 0 classical, 1 direct
    smoother: int = SMOOTH_GS
    pre_smooth: int = 2
    post_smooth: int = 2
    relaxation: float = 1.0
    strength_threshold: float = 0.25
    coarse_solve: int = COARSE_SWEEPS
    coarse_sweeps: int = 10
    aggregate_size: int = 8
    seed: int = 0
    coarse_order: int = 0  # 0 selection order (reference), 1 ascending fine index
    max_interp_points: int = 0  # 0: every interpolation weight (the reference)

    def _c(self):
        return _AmgConfig(self.max_levels, self.coarsening, self.min_coarse_size, self.interpolation,
                          self.smoother, self.pre_smooth, self.post_smooth, self.relaxation,
                          self.strength_threshold, self.coarse_solve, self.coarse_sweeps,
                          self.aggregate_size, self.seed, self.coarse_order, self.max_interp_points)


class Amg:
    def __init__(self, a: Csr, cfg: AmgConfig):
        self._a = a
        self.cfg = cfg
        c = cfg._c()
        self.h = lib().or_amg_setup(a.h, C.byref(c))

    @classmethod
    def from_levels(cls, levels, cfg: AmgConfig):
        """levels: [[A_0, P_0, R_0], ..., [A_L]] of Csr."""
        obj = cls.__new__(cls)
        nl = len(levels)
        arr = C.c_void_p * nl
        A = arr(*[lv[0].h for lv in levels])
        Pm = arr(*[lv[1].h if len(lv) > 1 else None for lv in levels])
        R = arr(*[lv[2].h if len(lv) > 1 else None for lv in levels])
        obj._a = levels
        obj.cfg = cfg
        c = cfg._c()
        obj.h = lib().or_amg_from_levels(nl, A, Pm, R, C.byref(c))
        return obj

    @property
    def num_levels(self):
        return lib().or_amg_num_levels(self.h)

    def level(self, l, which=0):
        p = lib().or_amg_level(self.h, l, which)
        return Csr(p, owned=False) if p else None

    def apply(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.empty_like(r)
        lib().or_amg_apply(self.h, _ptr(r), _ptr(z))
        return z

    def operator_complexity(self):
        tot = sum(self.level(l).info()[2] for l in range(self.num_levels))
        return tot / self.level(0).info()[2]

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_amg_free(self.h)
            self.h = None


@dataclass
class Report:
    termination: str
    iterations: int
    initial_residual: float
    final_residual: float
    threshold: float
    history: np.ndarray


def _krylov(fn, a: Csr, b, x0=None, precond=PRE_NONE, amg: Amg | None = None, tol=0.0, rtol=1e-8,
            max_it=1000):
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
    cfg = _SolverConfig(tol, rtol, max_it)
    rep = _Report()
    hist = np.full(max_it + 1, np.nan)
    rc = fn(a.h, precond, amg.h if amg is not None else None, _ptr(b), _ptr(x), C.byref(cfg),
            C.byref(rep), _ptr(hist))
    if rc != 0:
        raise ValueError(f"oracle solve setup failed ({rc})")
    return x, Report(TERMINATIONS[rep.termination], rep.iterations, rep.initial_residual,
                     rep.final_residual, rep.threshold, hist[: rep.iterations + 1])


def pcg(a, b, **kw):
    return _krylov(lib().or_pcg, a, b, **kw)


def bicgstab(a, b, **kw):
    return _krylov(lib().or_bicgstab, a, b, **kw)


def gmres(a: Csr, b, restart=30, **kw):
    """Restarted right-preconditioned GMRES(m), m from the restart ladder."""
    fn = lib().or_gmres

    def call(h, pre, amg, bp, xp, cfg, rep, hist):
        return fn(h, pre, amg, restart, bp, xp, cfg, rep, hist)
    return _krylov(call, a, b, **kw)


def gmres_width(requested: int) -> int:
    return lib().or_gmres_width(requested)


def pcg_equilibrated(a: Csr, b, x0=None, tol=0.0, rtol=1e-10, max_it=20000):
    """Jacobi-PCG with the 1-D solver's row-equilibrated residual test."""
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
    cfg = _SolverConfig(tol, rtol, max_it)
    rep = _Report()
    rc = lib().or_pcg_equilibrated(a.h, _ptr(b), _ptr(x), C.byref(cfg), C.byref(rep))
    if rc != 0:
        raise ValueError(f"oracle solve setup failed ({rc})")
    return x, Report(TERMINATIONS[rep.termination], rep.iterations, rep.initial_residual, rep.final_residual,
                     rep.threshold, np.zeros(0))


LS_CG, LS_BICGSTAB, LS_DETECT = 0, 1, 2
LS_PATHS = ["krylov", "direct", "direct_unscaled", "krylov_fallback", "failed", "error"]


class _LsReport(C.Structure):
    _fields_ = [("method", C.c_int32), ("path", C.c_int32), ("termination", C.c_int32), ("pad", C.c_int32),
                ("iterations", C.c_int64), ("residual", C.c_double)]


@dataclass
class LsReport:
    method: int       # LS_CG or LS_BICGSTAB
    path: str         # one of LS_PATHS
    termination: str  # of the Krylov solve, "" when none ran
    iterations: int
    residual: float   # ||D (A x - b)|| / ||D b||


def detect_solver_method(a: Csr) -> int:
    """NetworkSolver::detect_solver_method: LS_CG or LS_BICGSTAB."""
    return lib().or_detect_solver_method(a.h)


def dense_lu_solve(m: np.ndarray, b):
    """Dense LU with partial pivoting; None on a zero pivot."""
    mm = np.array(m, dtype=np.float64, order="C")
    bb = np.array(b, dtype=np.float64)
    return bb if lib().or_dense_lu_solve(mm.shape[0], _ptr(mm), _ptr(bb)) == 0 else None


def linear_system_solve(a: Csr, b, x0=None, method=LS_DETECT, tolerance=1e-10, max_iterations=20000):
    """LinearSystemSolver::solve_with_initial_guess of the 1-D network solver."""
    n = a.info()[0]
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    rep = _LsReport()
    if lib().or_linear_system_solve(a.h, _ptr(b), _ptr(x), method, tolerance, max_iterations, C.byref(rep)) != 0:
        raise ValueError("linear_system_solve: matrix is not square")
    term = TERMINATIONS[rep.termination] if rep.termination >= 0 else ""
    return x, LsReport(rep.method, LS_PATHS[rep.path], term, rep.iterations, rep.residual)


def set_threads(n: int):
    lib().or_set_threads(n)


def get_threads() -> int:
    return lib().or_get_threads()


NETWORK_ERRORS = {1: "self-loop edge", 2: "non-finite conductance", 3: "non-positive conductance"}


def network_assemble(n_nodes, edges_i, edges_j, conductance, fixed, fixed_value, neumann=None):
    """The grounded conductance Laplacian and right-hand side of one network
    (``or_network_assemble``). ``fixed`` is a per-node 0/1 mask of Dirichlet
    nodes and ``fixed_value`` their pressures. Returns ``(Csr, rhs)``; raises
    ``ValueError`` naming the first offending edge as the reference does."""
    n = int(n_nodes)
    ei = np.ascontiguousarray(edges_i, dtype=np.int64)
    ej = np.ascontiguousarray(edges_j, dtype=np.int64)
    g = np.ascontiguousarray(conductance, dtype=np.float64)
    fx = np.ascontiguousarray(fixed, dtype=np.int8)
    fv = np.ascontiguousarray(fixed_value, dtype=np.float64)
    q = None if neumann is None else np.ascontiguousarray(neumann, dtype=np.float64)
    rhs = np.zeros(n)
    out = C.c_void_p()
    bad = C.c_int64()
    rc = lib().or_network_assemble(n, ei.shape[0], _ptr(ei), _ptr(ej), _ptr(g), _ptr(fx), _ptr(fv),
                                   None if q is None else _ptr(q), C.byref(out), _ptr(rhs), C.byref(bad))
    if rc != 0:
        raise ValueError(f"{NETWORK_ERRORS[rc]} at edge {bad.value}")
    return Csr(out.value), rhs


class Simple:
    """SimplePreconditioner of a saddle-point matrix whose first ``n_velocity``
    unknowns are velocities (``or_simple_new``)."""

    def __init__(self, a: Csr, n_velocity: int):
        self.h = lib().or_simple_new(a.h, int(n_velocity))
        if not self.h:
            raise ValueError("SIMPLE needs a square matrix and 0 <= n_velocity <= n")
        self.n = a.info()[0]

    def apply(self, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n)
        lib().or_simple_apply(self.h, _ptr(b), _ptr(x))
        return x

    def apply_block_diagonal(self, b):
        """BlockDiagonalPreconditioner of the same split."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n)
        lib().or_block_diagonal_apply(self.h, _ptr(b), _ptr(x))
        return x

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_simple_free(self.h)
            self.h = None


PRE_SIMPLE, PRE_BLOCK_DIAGONAL = 3, 4


def gmres_simple(a: Csr, simple: Simple, b, restart=30, precond=PRE_SIMPLE, **kw):
    """GMRES(m) right-preconditioned by SIMPLE, or with ``precond =
    PRE_BLOCK_DIAGONAL`` by the block diagonal of the same split
    (``or_gmres_saddle``)."""
    fn = lib().or_gmres_saddle

    def call(h, pre, amg, bp, xp, cfg, rep, hist):
        return fn(h, simple.h, precond, restart, bp, xp, cfg, rep, hist)
    return _krylov(call, a, b, **kw)


class ComponentBlock:
    """ComponentBlockPreconditioner (block_preconditioner.rs:609-976) on the
    oracle; ValueError with the reason code when the reference's constructor
    would return Err (1 split, 2 component coupling, 3 singular block)."""

    def __init__(self, a: Csr, n_velocity: int, pivot_tolerance: float = 1e-12):
        err = C.c_int(0)
        self.h = lib().or_component_block_new(a.h, n_velocity, pivot_tolerance, C.byref(err))
        self.n = a.info()[0]
        if not self.h:
            raise ValueError(f"component-block setup refused ({err.value})")

    def apply(self, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n)
        lib().or_component_block_apply(self.h, _ptr(b), _ptr(x))
        return x

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_component_block_free(self.h)
            self.h = None


def gmres_component_block(a: Csr, cb: ComponentBlock, b, restart=30, **kw):
    def call(h, pre, amg, bp, xp, cfg, rep, hist):
        return lib().or_gmres_component_block(h, cb.h, restart, bp, xp, cfg, rep, hist)
    return _krylov(call, a, b, **kw)
