/*
 * CPU oracle for the CFDrs preconditioned sparse linear-solve path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the oracle used by tests/,
 * __graft_entry__.smoke() and the CPU-baseline leg of bench.py. The product
 * library (cfdrs_b200/libcfdgpu.so) never links, loads or calls it.
 *
 * It restates, in plain C++17/OpenMP, the FP64 algorithms of the reference
 * (ryancinsight/CFDrs, Rust) for this path:
 *   - CSR SpMV                      leto_ops::spmv_into via crates/cfd-math/src/sparse/operations.rs:50-79
 *   - strength of connection        crates/cfd-math/src/linear_solver/preconditioners/multigrid/coarsening/algorithms.rs:395-436
 *   - Ruge-Stueben C/F split        .../coarsening/algorithms.rs:34-126 (+ assign_closest_coarse_points :199-230)
 *   - aggregation / PMIS            .../coarsening/algorithms.rs:129-172, :310-354 (PMIS priorities seeded)
 *   - classical / direct interp.    .../multigrid/interpolation.rs:38-188, :191-217
 *   - Galerkin RAP, R = P^T         .../multigrid/amg.rs:290-380
 *   - V-cycle                       .../multigrid/amg.rs:423-503, entry with z = 0 at :553-554
 *   - Jacobi / GS / SGS smoothers   .../multigrid/smoothers.rs:45-199
 *   - Jacobi preconditioner         crates/cfd-1d/src/solver/core/linear_system.rs:270-332
 *   - PCG / BiCGSTAB + termination  crates/cfd-math/src/linear_solver/krylov.rs:253-360, :375-428
 *     (the recurrences themselves live in the un-vendored athena-core 0.1.1 @ f6608bef;
 *      they are restated from Saad 2003, Alg. 9.1 / 7.7, which the reference cites).
 *
 * Parity is pinned by the golden vectors transcribed from the reference's own
 * unit tests (tests/golden/make_golden.py lists each with its file:line).
 */
#ifndef CFD_ORACLE_H
#define CFD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_csr or_csr;
typedef struct or_amg or_amg;

/* CSR matrices (int64 indices mirror the reference's usize). */
or_csr* or_csr_new(int64_t nrows, int64_t ncols, int64_t nnz, const int64_t* row_ptr,
                   const int64_t* col, const double* val);
void or_csr_info(const or_csr* a, int64_t* nrows, int64_t* ncols, int64_t* nnz);
void or_csr_export(const or_csr* a, int64_t* row_ptr, int64_t* col, double* val);
void or_csr_free(or_csr* a);

void or_set_threads(int n);
int or_get_threads(void);

void or_spmv(const or_csr* a, const double* x, double* y);
or_csr* or_strength(const or_csr* a, double theta);
or_csr* or_transpose(const or_csr* a);
or_csr* or_spgemm(const or_csr* a, const or_csr* b);

/* Coarsening kinds. */
enum { OR_RUGE_STUEBEN = 0, OR_AGGREGATION = 1, OR_PMIS = 2 };
/* Returns the number of coarse points; coarse_points[0..nc) in selection order,
 * f2c[i] = coarse index or -1. literal_scan=1 uses the reference's O(n^2) scan
 * for the Ruge-Stueben maximum (for pinning the fast path on small inputs). */
int64_t or_coarsen(const or_csr* a, int kind, double theta, int64_t param, uint64_t seed,
                   int literal_scan, int64_t* coarse_points, int64_t* f2c);
or_csr* or_classical_interp(const or_csr* a, const int64_t* coarse_points, int64_t nc,
                            const or_csr* strength);
or_csr* or_direct_interp(const int64_t* f2c, int64_t n, int64_t nc);

enum { OR_SMOOTH_JACOBI = 0, OR_SMOOTH_GS = 1, OR_SMOOTH_SGS = 2 };
void or_smooth(const or_csr* a, double* x, const double* b, int kind, double omega, int iters);

/* Dense LU with partial pivoting solve of a small CSR system (coarsest level). */
int or_dense_solve(const or_csr* a, const double* b, double* x);

enum { OR_COARSE_SWEEPS = 0, OR_COARSE_DENSE = 1 };
typedef struct {
  int32_t max_levels;
  int32_t coarsening;      /* OR_RUGE_STUEBEN ... */
  int64_t min_coarse_size;
  int32_t interpolation;   /* 0 classical (reference), 1 direct, 2 modified classical */
  int32_t smoother;        /* OR_SMOOTH_* */
  int32_t pre_smooth;
  int32_t post_smooth;
  double relaxation;
  double strength_threshold;
  int32_t coarse_solve;    /* OR_COARSE_* */
  int32_t coarse_sweeps;   /* reference: 10 */
  int64_t aggregate_size;  /* reference: 8 */
  uint64_t seed;           /* PMIS priorities */
  int32_t coarse_order;    /* 0 selection order (reference), 1 ascending fine index */
  int32_t max_interp_points; /* 0: every weight (the reference ignores the argument, interpolation.rs:42);
                                k: the k largest-magnitude weights per row, rescaled to the row sum */
} or_amg_config;

or_amg* or_amg_setup(const or_csr* a, const or_amg_config* cfg);
or_amg* or_amg_from_levels(int nlev, const or_csr* const* a, const or_csr* const* p,
                           const or_csr* const* r, const or_amg_config* cfg);
int or_amg_num_levels(const or_amg* h);
/* which: 0 = A_l, 1 = P_l (interpolation), 2 = R_l (restriction). NULL when absent. */
const or_csr* or_amg_level(const or_amg* h, int level, int which);
void or_amg_apply(const or_amg* h, const double* r, double* z);
void or_amg_free(or_amg* h);

/* Krylov. */
enum { OR_PRE_NONE = 0, OR_PRE_JACOBI = 1, OR_PRE_AMG = 2, OR_PRE_SIMPLE = 3, OR_PRE_BLOCK_DIAGONAL = 4,
       OR_PRE_COMPONENT_BLOCK = 5 };
enum {
  OR_TERM_CONVERGED = 0,
  OR_TERM_INITIAL_RESIDUAL = 1,
  OR_TERM_MAX_ITERATIONS = 2,
  OR_TERM_BREAKDOWN = 3,
  OR_TERM_NON_POSITIVE_CURVATURE = 4
};
typedef struct {
  double tolerance;           /* absolute */
  double relative_tolerance;  /* relative to ||r0|| */
  int64_t max_iterations;
} or_solver_config;
typedef struct {
  int32_t termination;
  int32_t pad;
  int64_t iterations;
  double initial_residual;
  double final_residual;
  double threshold;
} or_report;

/* Return 0 on success, <0 on a setup/dimension error (e.g. non-finite diagonal). */
int or_pcg(const or_csr* a, int precond, const or_amg* amg, const double* b, double* x,
           const or_solver_config* cfg, or_report* rep, double* history);
int or_pcg_equilibrated(const or_csr* a, const double* b, double* x, const or_solver_config* cfg,
                        or_report* rep);
int or_bicgstab(const or_csr* a, int precond, const or_amg* amg, const double* b, double* x,
                const or_solver_config* cfg, or_report* rep, double* history);
/* Restart width actually used for a requested restart (the ladder of krylov.rs:96-120). */
int or_gmres_width(int64_t requested);
/* Restarted right-preconditioned GMRES(m); history[k] = implicit residual after k steps. */
int or_gmres(const or_csr* a, int precond, const or_amg* amg, int64_t restart, const double* b, double* x,
             const or_solver_config* cfg, or_report* rep, double* history);

/* SIMPLE saddle-point preconditioner (crates/cfd-math/src/linear_solver/
 * block_preconditioner.rs:400-568): the first n_velocity unknowns are
 * velocities, the rest pressures. NULL for a non-square matrix or an
 * n_velocity outside [0, n]. */
typedef struct or_simple or_simple;
or_simple* or_simple_new(const or_csr* a, int64_t n_velocity);
void or_simple_apply(const or_simple* s, const double* b, double* x);
void or_simple_free(or_simple* s);
/* BlockDiagonalPreconditioner (block_preconditioner.rs:189-398) of the same
 * split: x = b * its inverse diagonal. */
void or_block_diagonal_apply(const or_simple* s, const double* b, double* x);
/* ComponentBlockPreconditioner (block_preconditioner.rs:609-976, the GMRES +
 * ComponentBlock tier of chain.rs:193-217): the velocity block of a 3-D
 * saddle system is component-major, three equal components; each component
 * block (cross-component velocity entries above 1e-14 are refused) gets its
 * zero diagonals stabilized and an exact factorization (dense LU with partial
 * pivoting here; the reference's provider sparse LU is not vendored: both are
 * exact solves), the pressure Schur approximation C - D diag(A)^-1 G is
 * assembled, stabilized and lumped by signed row sums. Apply (the athena
 * path, :920-975): u* = A_c^-1 r_u per component, p = lumped^-1 (r_p - D u*),
 * u = u* - A_c^-1 (G p) per component. NULL (with *error set) when the split
 * is not 3 equal components, a cross-component entry exceeds 1e-14, or a
 * block is singular. pivot_tolerance: the stabilization scale of the
 * provider's sparse LU (not vendored; the tests pass 1e-12). */
typedef struct or_component_block or_component_block;
or_component_block* or_component_block_new(const or_csr* a, int64_t n_velocity, double pivot_tolerance,
                                           int* error);
void or_component_block_apply(const or_component_block* c, const double* r, double* z);
void or_component_block_free(or_component_block* c);
int or_gmres_component_block(const or_csr* a, const or_component_block* c, int64_t restart, const double* b,
                             double* x, const or_solver_config* cfg, or_report* rep, double* history);

/* GMRES(m) right-preconditioned by SIMPLE (precond OR_PRE_SIMPLE,
 * chain.rs:216-238) or by the block diagonal (OR_PRE_BLOCK_DIAGONAL,
 * chain.rs:265-285) of the split. */
int or_gmres_saddle(const or_csr* a, const or_simple* simple, int precond, int64_t restart, const double* b,
                    double* x, const or_solver_config* cfg, or_report* rep, double* history);

/* The 1-D network solve, LinearSystemSolver::solve_with_initial_guess
 * (crates/cfd-1d/src/solver/core/linear_system.rs:114-155) with the method of
 * NetworkSolver::detect_solver_method (solver_detection.rs:36-64):
 *   - rows equilibrated by 1 / max_j |a_ij| (identity where that maximum is not
 *     above f64::EPSILON or not finite, :157-186);
 *   - n <= 256: dense LU of the equilibrated system, kept if it meets the
 *     residual target on the original system (:188-204), else dense LU of
 *     the original system (:124-130);
 *   - n > 256: CG or BiCGSTAB on the equilibrated system with DiagJacobi of
 *     it, IterativeSolverConfig::new(tol) (absolute tolerance tol on the
 *     2-norm of its residual, max_iterations), x in as the initial guess; kept
 *     if converged and the residual target holds, else dense LU of the
 *     original system (:131-155).
 * Dense LU: partial pivoting (first largest |a_ik| in row order), fails on a
 * zero or non-finite pivot; the reference then tries a QR least-squares solve
 * (:248-267), which is not restated: the system is reported failed. */
enum { OR_LS_CG = 0, OR_LS_BICGSTAB = 1, OR_LS_DETECT = 2 };
enum {
  OR_LS_PATH_KRYLOV = 0,          /* the Krylov solution was kept */
  OR_LS_PATH_DIRECT = 1,          /* dense LU of the equilibrated system */
  OR_LS_PATH_DIRECT_UNSCALED = 2, /* dense LU of the original system after the first missed the target */
  OR_LS_PATH_KRYLOV_FALLBACK = 3, /* dense LU of the original system after the Krylov solve */
  OR_LS_PATH_FAILED = 4,          /* the last dense LU met a zero pivot */
  OR_LS_PATH_ERROR = 5            /* DiagJacobi::new refused a non-finite diagonal (an Err) */
};
typedef struct {
  int32_t method;       /* OR_LS_CG or OR_LS_BICGSTAB (the detected one under OR_LS_DETECT) */
  int32_t path;         /* OR_LS_PATH_* */
  int32_t termination;  /* of the Krylov solve (OR_TERM_*), -1 when none ran */
  int32_t pad;
  int64_t iterations;   /* Krylov iterations */
  double residual;      /* ||D (A x - b)|| / ||D b|| of the returned x (the target test's ratio) */
} or_ls_report;
/* NetworkSolver::detect_solver_method: OR_LS_CG or OR_LS_BICGSTAB. */
int or_detect_solver_method(const or_csr* a);
/* Dense LU with partial pivoting of the row-major n x n matrix m (overwritten),
 * solving m x = b in place of b. 0, or -1 on a zero or non-finite pivot. */
int or_dense_lu_solve(int64_t n, double* m, double* b);
/* x holds the initial guess in and the solution out. Returns 0, or -1 for a
 * non-square matrix. */
int or_linear_system_solve(const or_csr* a, const double* b, double* x, int method, double tolerance,
                           int64_t max_iterations, or_ls_report* rep);

/* MatrixAssembler::assemble_into for one network (crates/cfd-1d/src/solver/core/
 * matrix_assembly.rs:163-250). Nodes 0..n-1, edges (ei[e], ej[e]) with
 * conductance g[e]; fixed[k] != 0 marks a Dirichlet node of pressure
 * fixed_value[k]; neumann may be NULL. Returns 0 and a new CSR in *out with the
 * right-hand side in rhs[n]; 1 self-loop, 2 non-finite conductance, 3
 * non-positive conductance, with the edge in *bad_edge. */
int or_network_assemble(int64_t n, int64_t m, const int64_t* ei, const int64_t* ej, const double* g,
                        const int8_t* fixed, const double* fixed_value, const double* neumann, or_csr** out,
                        double* rhs, int64_t* bad_edge);

#ifdef __cplusplus
}
#endif
#endif
