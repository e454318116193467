/*
 * cfdgpu.h -- C ABI of the B200 (sm_100a) sparse linear-solve library that
 * stands in for cfd-math's Krylov / preconditioner surface of CFDrs.
 *
 * Plain pointers and sizes only. Every entry point returns a cfd_status; a
 * human-readable message for the last failure on the calling thread is
 * available from cfd_last_error(). Numerical end states (converged, stalled,
 * broken down) are NOT errors: they are reported in cfd_solve_report, as the
 * reference reports them value-semantically (krylov.rs:362-401).
 *
 * Reference interfaces replaced (paths relative to the CFDrs repository):
 *   cfd_solve                krylov::cg_preconditioned       crates/cfd-math/src/linear_solver/krylov.rs:318-343
 *                            krylov::bicgstab_preconditioned  krylov.rs:253-278
 *                            krylov::gmres_preconditioned     krylov.rs:150-221 (gmres :228-246)
 *                            krylov::cg / krylov::bicgstab    krylov.rs:350-360 / :285-308
 *                            SolverKind::solve[_preconditioned] krylov.rs:562-612
 *   cfd_solver_config        IterativeSolverConfig -> convergence_policy, krylov.rs:123-139
 *   cfd_solve_report         athena SolveReport{termination, iterations, initial_residual_norm,
 *                            final_residual_norm, threshold} (fields read at krylov.rs:486, 509-512)
 *   cfd_termination          athena Termination as mapped by krylov::interpret, krylov.rs:385-399
 *   cfd_csr_create           leto_ops::CsrMatrix::from_parts (e.g. krylov.rs:467), the borrowed
 *                            BorrowedCsrOperator of krylov.rs:330
 *   cfd_csr_update_values    same pattern, new values (the input of AlgebraicMultigrid::recompute)
 *   cfd_spmv                 leto_ops::spmv_into, wrapped at crates/cfd-math/src/sparse/operations.rs:50-79
 *   cfd_amg_config           AMGConfig, crates/cfd-math/src/linear_solver/preconditioners/multigrid/mod.rs:219-259
 *   cfd_amg_setup            AlgebraicMultigrid::new, .../multigrid/amg.rs:133-146
 *   cfd_amg_recompute        AlgebraicMultigrid::recompute, amg.rs:179-214
 *   cfd_amg_apply            Preconditioner::apply_to (z = 0, one V-cycle), amg.rs:507-557
 *   cfd_amg_stats            AMGStatistics, multigrid/mod.rs:366-395
 *   cfd_jacobi_*             DiagJacobi, crates/cfd-1d/src/solver/core/linear_system.rs:270-332
 *   cfd_batch_linear_system_solve
 *                            LinearSystemSolver::solve_with_initial_guess called once per network
 *                            (crates/cfd-1d/src/solver/core/linear_system.rs:114-155) by the
 *                            cfd-optim candidate fold (crates/cfd-optim/src/metrics/blueprint_graph.rs:48-135)
 *   cfd_batch_solve          krylov::cg_preconditioned with DiagJacobi per system (krylov.rs:318-343,
 *                            linear_system.rs:270-332), stopping on the 1-D solver's equilibrated residual
 *   cfd_adjoint_*            no reference counterpart (new differentiable-solve layer; see each entry)
 */
#ifndef CFDGPU_H
#define CFDGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status / termination -------------------------------------------- */
typedef enum {
  CFD_OK = 0,
  CFD_ERR_DIM = 1,       /* dimension / structure mismatch (Error::InvalidConfiguration) */
  CFD_ERR_CONFIG = 2,    /* invalid solver / AMG configuration (convergence_policy rejection) */
  CFD_ERR_CUDA = 3,      /* CUDA runtime failure */
  CFD_ERR_TIMEOUT = 4,   /* a bounded device wait ran out */
  CFD_ERR_NONFINITE = 5, /* non-finite input (e.g. DiagJacobi::new on a non-finite diagonal) */
  CFD_ERR_ALLOC = 6,     /* device or host allocation failed */
  CFD_ERR_STATE = 7      /* handle used in the wrong state (e.g. recompute before setup) */
} cfd_status;

typedef enum {
  CFD_TERM_CONVERGED = 0,
  CFD_TERM_INITIAL_RESIDUAL = 1,
  CFD_TERM_MAX_ITERATIONS = 2,        /* SolveOutcome::Stalled */
  CFD_TERM_BREAKDOWN = 3,             /* SolveOutcome::BrokenDown */
  CFD_TERM_NON_POSITIVE_CURVATURE = 4 /* SolveOutcome::BrokenDown */
} cfd_termination;

const char* cfd_last_error(void);
const char* cfd_version(void);

/* ---- context: one device + one stream ---------------------------------- */
typedef struct cfd_context cfd_context;
cfd_status cfd_context_create(int device, cfd_context** out);
/* Run subsequent work of this context on an existing stream (e.g. torch's
 * current stream); NULL restores the context's own stream. To run on CUDA's
 * legacy default stream pass cudaStreamLegacy ((void*)0x1). */
cfd_status cfd_context_set_stream(cfd_context* ctx, void* cuda_stream);
/* FP64 CG and Jacobi-PCG (cfd_solve) of a system whose rows fit the shared
 * memory of one thread-block cluster (up to 16 CTAs; e.g. 16 384 rows of a
 * 5-point operator) run as one launch, the whole recurrence on chip
 * (enable != 0, the default); 0 keeps the multi-kernel solve for every size.
 * Same recurrence and termination; the dot products sum in another order. */
cfd_status cfd_context_set_cluster_solve(cfd_context* ctx, int32_t enable);
cfd_status cfd_context_synchronize(cfd_context* ctx);
cfd_status cfd_context_destroy(cfd_context* ctx);

/* ---- device CSR -------------------------------------------------------- */
typedef struct cfd_csr cfd_csr;
/* Host arrays (row_ptr[nrows+1], col[nnz] sorted per row, val[nnz]); copied to
 * the device. Indices must fit int32. */
cfd_status cfd_csr_create(cfd_context* ctx, int64_t nrows, int64_t ncols, int64_t nnz,
                          const int64_t* row_ptr, const int64_t* col, const double* val,
                          cfd_csr** out);
cfd_status cfd_csr_create_i32(cfd_context* ctx, int64_t nrows, int64_t ncols, int64_t nnz,
                              const int64_t* row_ptr, const int32_t* col, const double* val,
                              cfd_csr** out);
cfd_status cfd_csr_update_values(cfd_csr* a, const double* val_host);
cfd_status cfd_csr_info(const cfd_csr* a, int64_t* nrows, int64_t* ncols, int64_t* nnz);
cfd_status cfd_csr_destroy(cfd_csr* a);

/* ---- SpMV device layout (no reference counterpart: CFDrs multiplies plain
 * CSR, crates/cfd-math/src/sparse/operations.rs:14-30) -------------------
 * Row blocks of <= 512 rows / 4096 nonzeros. A block whose column offsets from
 * base(row) = row * ncols / nrows take <= 256 values stores one-byte codes;
 * when every block is coded and its columns fall in <= 8 windows of <= 4096
 * entries in total, SpMV stages those x windows in shared memory ("x staged"). */
typedef struct {
  int64_t blocks;
  int64_t compressed_nnz;    /* nonzeros stored as one-byte codes */
  int32_t all_compressed;
  int32_t x_staged;
  int32_t threads_per_row;
  int32_t max_windows;       /* cfd_layout_check only */
  int64_t staged_x_entries;  /* cfd_layout_check only: x entries staged over all blocks */
  int32_t path_f32;          /* SpMV pipeline an SpMV runs per precision (cfd_spmv_path; TIMED until timed) */
  int32_t path_f64;
  int32_t sliced;            /* the sliced layout (CFD_PATH_SLICED) is built */
  int32_t diagonals;         /* stored diagonals of the diagonal layout (CFD_PATH_DIAGONAL), 0 when none */
  int64_t sliced_slots;      /* its slots (stored nonzeros plus padding) */
} cfd_layout_info;
cfd_status cfd_csr_layout(const cfd_csr* a, cfd_layout_info* out);
/* SpMV pipelines. All sum every row in the same order, so y = A x is identical
 * on each; dot products fused into solver SpMVs add per-CTA partials over each
 * pipeline's own grid (deterministic for a pipeline, equal to rounding across
 * pipelines). SPLIT takes any matrix, RECORD needs every block coded (otherwise it
 * runs as SPLIT), X_STAGED needs x staging and a 16-byte aligned x (otherwise
 * it runs as RECORD). SLICED (FP32 only) needs the sliced layout: one thread
 * per row, rows of at most 32 entries in slices of 32 rows padded by at most
 * 15 %, at most 255 column offsets per 512 rows (otherwise it runs as RECORD).
 * DIAGONAL needs the diagonal layout: a square matrix, one thread per row,
 * every entry on one of at most 8 diagonals (column - row) with at most 10 %
 * empty slots (stencil operators); values stored diagonal-major, no indices.
 * It adds an empty slot as 0 * x, identical to skipping it for finite x.
 * AUTO (the default): DIAGONAL when eligible (on the 256^3 7-point operator
 * it beats the record and x-staged pipelines in both precisions); otherwise
 * RECORD for FP32 (SLICED runs the plain SpMV as fast and the fused epilogues
 * slower), X_STAGED for FP64 when eligible with one thread per row, SPLIT
 * otherwise. TIMED: at the
 * next SpMV in that precision, time the eligible pipelines (allocates scratch
 * vectors) and keep the fastest. */
typedef enum {
  CFD_PATH_TIMED = -2,
  CFD_PATH_AUTO = -1,
  CFD_PATH_SPLIT = 0,
  CFD_PATH_RECORD = 1,
  CFD_PATH_X_STAGED = 2,
  CFD_PATH_SLICED = 3,
  CFD_PATH_DIAGONAL = 4
} cfd_spmv_path;
/* Set the pipeline of one precision (fp32 != 0: FP32 values). CFD_ERR_CONFIG
 * when the matrix is not eligible for it. */
cfd_status cfd_csr_set_path(cfd_csr* a, int32_t fp32, int32_t path);
/* Host only, no GPU: builds the layout of a CSR matrix and evaluates y = A x by
 * walking the device kernels' index arithmetic (staged x image, index record,
 * codes, tables), failing with CFD_ERR_STATE and a message on any index
 * outside its region. */
cfd_status cfd_layout_check(int64_t nrows, int64_t ncols, int64_t nnz, const int64_t* row_ptr,
                            const int32_t* col, const double* val, const double* x, double* y,
                            cfd_layout_info* out);

/* y = A x on device pointers (FP64), or FP32 values/vectors (values cast once). */
cfd_status cfd_spmv(cfd_csr* a, const double* x_dev, double* y_dev);
cfd_status cfd_spmv_f32(cfd_csr* a, const float* x_dev, float* y_dev);

/* ---- AMG preconditioner ------------------------------------------------ */
typedef enum { CFD_COARSEN_RUGE_STUEBEN = 0, CFD_COARSEN_AGGREGATION = 1, CFD_COARSEN_PMIS = 2 } cfd_coarsening;
/* CLASSICAL: the reference formula (interpolation.rs:38-188). MODIFIED_CLASSICAL:
 * sign-restricted distribution with lumping of F-neighbours that share no
 * C-point (robust on deep hierarchies). DIRECT: piecewise constant (:191-217). */
typedef enum {
  CFD_INTERP_CLASSICAL = 0,
  CFD_INTERP_DIRECT = 1,
  CFD_INTERP_MODIFIED_CLASSICAL = 2
} cfd_interpolation;
typedef enum { CFD_SMOOTH_JACOBI = 0 } cfd_smoother;
typedef enum { CFD_COARSE_SWEEPS = 0, CFD_COARSE_DENSE = 1 } cfd_coarse_solve;
/* SELECTION: coarse index = order of selection (the reference, algorithms.rs:81-85).
 * ASCENDING: coarse points numbered by ascending fine index -- the same
 * hierarchy up to a symmetric permutation per level (from level 2 on the
 * coarsening sees the permuted operator), with local P/R gathers. */
typedef enum { CFD_COARSE_ORDER_SELECTION = 0, CFD_COARSE_ORDER_ASCENDING = 1 } cfd_coarse_order;

typedef struct {
  int32_t max_levels;          /* AMGConfig::max_levels (default 10) */
  int32_t coarsening;          /* cfd_coarsening */
  int64_t min_coarse_size;     /* AMGConfig::min_coarse_size (default 50) */
  int32_t interpolation;       /* cfd_interpolation */
  int32_t smoother;            /* cfd_smoother (damped Jacobi only on the device) */
  int32_t pre_smooth;          /* AMGConfig::pre_smooth_iterations */
  int32_t post_smooth;         /* AMGConfig::post_smooth_iterations */
  double relaxation;           /* AMGConfig::relaxation_factor (omega) */
  double strength_threshold;   /* AMGConfig::strength_threshold (theta) */
  int32_t coarse_solve;        /* cfd_coarse_solve: reference sweeps (amg.rs:499-501) or dense FP64 */
  int32_t coarse_sweeps;       /* sweeps for CFD_COARSE_SWEEPS (reference: 10) */
  int64_t aggregate_size;      /* aggregation coarsening (reference passes 8, amg.rs:304) */
  uint64_t seed;               /* PMIS priorities (the reference draws them unseeded) */
  int32_t coarse_order;        /* cfd_coarse_order: numbering of each level's coarse points */
  /* The max_interpolation_points argument of create_classical_interpolation
   * (interpolation.rs:42), which the reference accepts and ignores: 0 keeps
   * every weight (the reference); k > 0 keeps the k weights of largest
   * magnitude in each row of P (ties: the smaller column), scaled so that the
   * row sum of P is unchanged. */
  int32_t max_interp_points;
} cfd_amg_config;

void cfd_amg_config_default(cfd_amg_config* cfg);

typedef struct {
  int32_t num_levels;
  int32_t pad;
  int64_t level_rows[16];
  int64_t level_nnz[16];
  double operator_complexity;
  double grid_complexity;
  double setup_seconds;
} cfd_amg_stats_t;

typedef struct cfd_amg cfd_amg;
cfd_status cfd_amg_setup(cfd_csr* a, const cfd_amg_config* cfg, cfd_amg** out);
/* New fine values of the setup's pattern (a on the hierarchy's context): the
 * Galerkin operators (R_l A_l) P_l, level diagonals, FP32 copies and the dense
 * coarsest inverse are re-formed on the device with P and R kept
 * (amg.rs:179-214), in the host product's summation order. CFD_ERR_DIM for
 * another pattern size, CFD_ERR_CONFIG for a singular coarsest operator
 * (CFD_COARSE_DENSE); the level operators then hold the new values while the
 * coarsest inverse is still the previous one, so recompute with nonsingular
 * values before the next apply or solve. */
cfd_status cfd_amg_recompute(cfd_amg* amg, cfd_csr* a);
/* z = M^-1 r (one V-cycle from z = 0), device pointers, FP64. */
cfd_status cfd_amg_apply(cfd_amg* amg, const double* r_dev, double* z_dev);
cfd_status cfd_amg_stats(const cfd_amg* amg, cfd_amg_stats_t* out);
/* The same hierarchy (AlgebraicMultigrid::setup, amg.rs:217-288, the host
 * part of cfd_amg_setup) built on the host only, from an n x n CSR with
 * int64 indices: no context, no device memory, no CUDA call. The handle
 * answers cfd_amg_stats, cfd_amg_level and cfd_amg_destroy; calls that need
 * the device return CFD_ERR_STATE. For callers that inspect or serialise the
 * hierarchy, and for checking the setup without a GPU. */
cfd_status cfd_amg_setup_host(int64_t n, const int64_t* row_ptr, const int64_t* col, const double* val,
                              const cfd_amg_config* cfg, cfd_amg** out);
/* SpMV pipeline of every level operator (A, P, R) in one precision, as
 * cfd_csr_set_path; an operator not eligible for the pipeline keeps AUTO.
 * No reference counterpart (CFDrs has one CSR SpMV). */
cfd_status cfd_amg_set_path(cfd_amg* amg, int32_t fp32, int32_t path);
/* Copy level `level`'s operator (which: 0 = A_l, 1 = P_l, 2 = R_l) to host
 * arrays; pass NULL arrays to query sizes only. After cfd_amg_recompute the
 * values of A_l are read back from the device on the first such call. */
cfd_status cfd_amg_level(const cfd_amg* amg, int level, int which, int64_t* nrows, int64_t* ncols,
                         int64_t* nnz, int64_t* row_ptr, int64_t* col, double* val);
cfd_status cfd_amg_destroy(cfd_amg* amg);

/* ---- Krylov solve ------------------------------------------------------ */
/* GMRES: restarted GMRES(m), right preconditioned, krylov::gmres_preconditioned
 * (krylov.rs:150-221); m = the requested restart rounded up the ladder 8, 16, 32,
 * 64, 128, 256 (RestartWidth::covering, krylov.rs:96-120), saturating at 256. */
typedef enum { CFD_SOLVER_CG = 0, CFD_SOLVER_BICGSTAB = 1, CFD_SOLVER_GMRES = 2 } cfd_solver_kind;
typedef enum {
  CFD_PRECOND_NONE = 0,
  CFD_PRECOND_JACOBI = 1,
  CFD_PRECOND_AMG = 2,
  CFD_PRECOND_SIMPLE = 3,         /* GMRES only; cfd_saddle_setup on the matrix first */
  CFD_PRECOND_BLOCK_DIAGONAL = 4, /* GMRES only; cfd_saddle_setup on the matrix first */
  CFD_PRECOND_COMPONENT_BLOCK = 5 /* GMRES only; cfd_component_block_setup on the matrix first */
} cfd_precond_kind;
typedef enum { CFD_PRECISION_FP64 = 0, CFD_PRECISION_FP32_REFINE = 1 } cfd_precision;
typedef enum { CFD_MEMORY_HOST = 0, CFD_MEMORY_DEVICE = 1 } cfd_memory;

typedef struct {
  double tolerance;           /* IterativeSolverConfig::tolerance (absolute) */
  double relative_tolerance;  /* IterativeSolverConfig::relative_tolerance (vs ||r0||) */
  int64_t max_iterations;     /* IterativeSolverConfig::max_iterations */
} cfd_solver_config;

typedef struct {
  int32_t solver;           /* cfd_solver_kind */
  int32_t precond;          /* cfd_precond_kind */
  int32_t precision;        /* cfd_precision */
  int32_t memory;           /* cfd_memory: b and x are host or device pointers */
  double inner_tolerance;   /* FP32 inner relative tolerance (refinement), e.g. 1e-4 */
  int32_t max_outer;        /* refinement steps cap */
  int32_t check_every;      /* device iterations between host convergence polls (0 = auto) */
  int32_t restart;          /* GMRES restart request (default 30, the pressure solver's GMRES(30)) */
} cfd_solve_options;

void cfd_solve_options_default(cfd_solve_options* opt);

typedef struct {
  int32_t termination;      /* cfd_termination */
  int32_t outer_iterations; /* refinement steps (0 for plain FP64) */
  int64_t iterations;       /* Krylov iterations (summed over refinement steps) */
  double initial_residual;  /* ||b - A x0||_2 */
  double final_residual;    /* FP64: recurrence residual; FP32_REFINE: true FP64 residual */
  double threshold;         /* max(tolerance, relative_tolerance * ||r0||) */
  double device_ms;         /* device time of the solve (CUDA events) */
} cfd_solve_report;

/* Solve A x = b; x carries the initial guess in and the solution out.
 * amg must be non-NULL when opt->precond == CFD_PRECOND_AMG. */
cfd_status cfd_solve(cfd_csr* a, const cfd_solve_options* opt, cfd_amg* amg, const double* b,
                     double* x, const cfd_solver_config* cfg, cfd_solve_report* rep);

/* ---- adjoint building blocks ------------------------------------------
 * No reference counterpart (CFDrs has no differentiable solve; its Python
 * layer crates/cfd-python/src/lib.rs:85-158 exposes physics solvers only).
 * For x = A^{-1} b and a loss L(x): lambda = A^{-T} dL/dx (for symmetric A a
 * second cfd_solve with the same preconditioner), dL/db = lambda and
 *   g[e] = dL/da_ij = -scale * lambda_i * x_j  for every stored entry e = (i, j).
 * All pointers are device pointers; g has nnz entries in A's CSR order. */
cfd_status cfd_pattern_outer(cfd_csr* a, const double* lambda_dev, const double* x_dev, double scale,
                             double* g_dev);
/* Replace A's values from device memory (same pattern); the host copy used by
 * AMG setup is refreshed too (cfd_amg_recompute reads the device values). */
cfd_status cfd_csr_set_values_device(cfd_csr* a, const double* val_dev);
/* The backward of x = A^-1 b for an upstream gradient g = dL/dx (device arrays
 * of n): lambda = A^-T g (dL/db), solved with opt (memory forced to device;
 * lambda starts from 0) on A when transpose == 0 (A symmetric: the forward's
 * preconditioner, AMG included, serves) or on A's transpose when transpose !=
 * 0 (formed from A's current values and kept until they change; Jacobi or no
 * preconditioner, e.g. BiCGSTAB for a non-symmetric A); then, when gvals is
 * not NULL, dL/da_ij = -lambda_i x_j on A's pattern into gvals (nnz). The
 * report is the transposed solve's. */
cfd_status cfd_adjoint(cfd_csr* a, const cfd_solve_options* opt, cfd_amg* amg, const double* x_dev,
                       const double* g_dev, double* lambda_dev, double* gvals_dev, int32_t transpose,
                       const cfd_solver_config* cfg, cfd_solve_report* rep);
/* The 2-D Darcy workload's assembly and its chain rule on the device, on the
 * context's stream. a holds the pattern of an n x n cell grid (row i + n j;
 * per row south, west, diagonal, east, north as present; checked once):
 * -div(exp(theta) grad p) = 0, harmonic-mean faces, p = 1 on the left and
 * p = 0 on the right wall at half a cell, no flux on top and bottom.
 * assemble: A's values (CSR order) and b from theta (n*n device arrays).
 * theta_grad: dL/dtheta from x = A^-1 b and lambda = A^-T dL/dx, the
 * face-coefficient chain rule in one kernel (no dL/dA array). CFD_ERR_DIM
 * when a is not that pattern. */
cfd_status cfd_darcy2d_assemble(cfd_csr* a, int64_t n, const double* theta_dev, double* val_dev, double* b_dev);
cfd_status cfd_darcy2d_theta_grad(cfd_csr* a, int64_t n, const double* theta_dev, const double* lambda_dev,
                                  const double* x_dev, double* grad_dev);

/* ---- saddle-point preconditioners -----------------------------------------
 * The two of LinearSolverChain's GMRES tiers for saddle-point systems
 * (crates/cfd-math/src/linear_solver/chain.rs:216-238, 265-285), over one
 * velocity/pressure split: the first n_velocity unknowns are velocities, the
 * rest pressures. cfd_saddle_setup builds both from the matrix's current
 * values; a later value update (cfd_csr_update_values,
 * cfd_csr_set_values_device) rebuilds them before the next use. Solve with
 * opt->solver = CFD_SOLVER_GMRES and opt->precond = CFD_PRECOND_SIMPLE or
 * CFD_PRECOND_BLOCK_DIAGONAL.
 * SIMPLE (SimplePreconditioner, block_preconditioner.rs:400-568): diag(A)^-1
 * (1 where |a_ii| <= 1e-14), the divergence rows D, the gradient block G and
 * diag(C - D diag(A)^-1 G)^-1; apply u* = diag(A)^-1 f, p = S^-1 (g - D u*),
 * u = u* - diag(A)^-1 G p.
 * Block diagonal (BlockDiagonalPreconditioner, :189-398): z = r / d with d the
 * momentum diagonal (1 where |a_ii| <= 1e-14) and, per pressure row, the
 * absolute row sum over the pressure block, or the mean |momentum diagonal|
 * where that sum is <= 1e-14. */
cfd_status cfd_saddle_setup(cfd_csr* a, int64_t n_velocity);
/* ComponentBlockPreconditioner (block_preconditioner.rs:609-976), the
 * preconditioner of LinearSolverChain's GMRES + ComponentBlock tier
 * (chain.rs:193-217), for 3-D saddle systems whose velocity block is
 * component-major: three equal components (n_velocity divisible by 3) with
 * no entry above 1e-14 coupling two components. Per component the block's
 * zero diagonals are stabilized (max(row scale * pivot_tolerance, 1e-14)
 * added, :71-107) and the block is solved exactly: the reference factors it
 * with its provider's sparse LU, this library forms the dense inverse on the
 * device (blocks of at most 8192 rows). The pressure Schur approximation
 * C - D diag(A)^-1 G is lumped by signed row sums (:112-137). Apply:
 * u* = A_c^-1 r_u, p = (r_p - D u*) / lumped, u = u* - A_c^-1 (G p).
 * CFD_ERR_DIM for a split that is not three equal components, CFD_ERR_CONFIG
 * for component coupling, an oversized or singular block (the reference's
 * constructor Errs there, and the chain skips the tier). A later value update
 * rebuilds it before the next use. */
cfd_status cfd_component_block_setup(cfd_csr* a, int64_t n_velocity, double pivot_tolerance);
/* z = M^-1 r on the device (FP64; r and z distinct device arrays of n). */
cfd_status cfd_component_block_apply(cfd_csr* a, const double* r_dev, double* z_dev);
/* z = M^-1 r on the device (FP64; r and z distinct device arrays of n). */
cfd_status cfd_simple_apply(cfd_csr* a, const double* r_dev, double* z_dev);
cfd_status cfd_block_diagonal_apply(cfd_csr* a, const double* r_dev, double* z_dev);
/* The same setup and apply on the host, for checks without a device. */
cfd_status cfd_simple_apply_host(int64_t n, const int64_t* row_ptr, const int32_t* col, const double* val,
                                 int64_t n_velocity, const double* b, double* x);
/* The block-diagonal inverse (n entries) on the host. */
cfd_status cfd_block_diagonal_host(int64_t n, const int64_t* row_ptr, const int32_t* col, const double* val,
                                   int64_t n_velocity, double* inv_diag);

/* ---- batched small systems --------------------------------------------
 * Many independent systems (e.g. the Kirchhoff networks of many design
 * candidates, solved one per call by the cfd-optim candidate fold,
 * crates/cfd-optim/src/metrics/blueprint_graph.rs:48-135). cfd_batch_solve:
 * Jacobi-PCG (krylov::cg_preconditioned with DiagJacobi) on each system as
 * given, in one persistent launch per size bucket replayed from a captured
 * CUDA graph. cfd_batch_linear_system_solve (below): the 1-D solver's full
 * cascade, LinearSystemSolver::solve_with_initial_guess
 * (crates/cfd-1d/src/solver/core/linear_system.rs:114-155).
 * Layout: system s owns global rows [sys_row_offsets[s], sys_row_offsets[s+1]);
 * row_ptr holds global nonzero offsets (total_rows + 1 entries); col holds the
 * column index LOCAL to the row's system. At most 2048 rows and 8192 nonzeros
 * per system. Convergence per system: the row-equilibrated residual
 * ||D(b - A x)|| <= max(tolerance, relative_tolerance * ||D(b - A x0)||),
 * D = 1 / max_j |a_ij| (linear_system.rs:157-204). */
typedef struct cfd_batch cfd_batch;
typedef struct {
  int32_t num_systems;
  int32_t converged_systems;
  int64_t total_iterations;   /* summed over systems (inner iterations for FP32_REFINE) */
  int32_t max_iterations;     /* largest per-system count */
  int32_t pad;
  double max_rel_residual;    /* largest final equilibrated relative residual */
  double device_ms;           /* copies in, graph, copies out (CUDA events) */
  /* cfd_batch_linear_system_solve only (0 otherwise), device time of its
   * phases: the dense solves of the systems of at most 256 rows, the Krylov
   * launches, and the dense fallback of the Krylov solves not kept. */
  double direct_ms, krylov_ms, fallback_ms;
} cfd_batch_report;
cfd_status cfd_batch_create(cfd_context* ctx, int32_t num_systems, const int64_t* sys_row_offsets,
                            const int64_t* row_ptr, const int32_t* col, const double* val,
                            cfd_batch** out);
cfd_status cfd_batch_update_values(cfd_batch* batch, const double* val_host);
/* opt: solver CG, precond JACOBI, precision FP64 or FP32_REFINE, memory of b/x.
 * x carries the initial guesses in and the solutions out. Per-system outputs
 * (host arrays of num_systems entries) may be NULL. b may be NULL after
 * cfd_batch_assemble: the assembled right-hand sides, resident on the device,
 * are used (a solve with a b of its own replaces them). */
cfd_status cfd_batch_solve(cfd_batch* batch, const cfd_solve_options* opt, const double* b, double* x,
                           const cfd_solver_config* cfg, int32_t* termination, int32_t* iterations,
                           double* rel_residual, cfd_batch_report* rep);
/* The 1-D network solve, LinearSystemSolver::solve_with_initial_guess
 * (crates/cfd-1d/src/solver/core/linear_system.rs:114-155), for every system
 * of the batch, with the method of NetworkSolver::detect_solver_method
 * (crates/cfd-1d/src/solver/core/solver_detection.rs:36-64) or a fixed one
 * (LinearSystemSolver::with_method). Per system:
 *   rows equilibrated by D = 1 / max_j |a_ij| (identity where that maximum is
 *   not above f64::EPSILON or not finite, linear_system.rs:157-186);
 *   n <= 256: dense LU (partial pivoting) of D A x = D b, kept when
 *   ||D (A x - b)|| <= tolerance * ||D b|| (:188-204), else dense LU of A x = b;
 *   n > 256: CG or BiCGSTAB on D A x = D b with DiagJacobi(D A) (identity where
 *   |d_ii| <= f64::EPSILON), IterativeSolverConfig::new(tolerance): stop at
 *   ||D b - D A x||_2 <= tolerance or after max_iterations; kept when it
 *   converged and the target above holds, else dense LU of A x = b.
 * Not restated: the QR least-squares solve the reference tries when a dense LU
 * meets a zero pivot; such a system is reported CFD_LS_PATH_FAILED. A
 * non-finite diagonal of D A (DiagJacobi::new's Err) is CFD_LS_PATH_ERROR.
 * FP32_REFINE runs the Krylov iterations in FP32 inside FP64 refinement of
 * the equilibrated system (the dense solves stay FP64). x carries the initial
 * guesses in and the solutions out; b may be NULL after cfd_batch_assemble.
 * results (num_systems entries, host) may be NULL. The dense solves use a
 * device scratch of one n x n FP64 matrix per CTA, allocated on first need
 * and kept by the batch. */
typedef enum { CFD_LS_CG = 0, CFD_LS_BICGSTAB = 1, CFD_LS_DETECT = 2 } cfd_ls_method;
typedef enum {
  CFD_LS_PATH_KRYLOV = 0,          /* the Krylov solution was kept */
  CFD_LS_PATH_DIRECT = 1,          /* dense LU of the equilibrated system (n <= 256) */
  CFD_LS_PATH_DIRECT_UNSCALED = 2, /* dense LU of A x = b after the first missed the target (n <= 256) */
  CFD_LS_PATH_KRYLOV_FALLBACK = 3, /* dense LU of A x = b after a Krylov solve that was not kept */
  CFD_LS_PATH_FAILED = 4,          /* the last dense LU met a zero pivot */
  CFD_LS_PATH_ERROR = 5            /* non-finite diagonal of D A */
} cfd_ls_path;
typedef struct {
  double tolerance;        /* LinearSystemSolver::with_tolerance (default 1e-6) */
  int64_t max_iterations;  /* LinearSystemSolver::with_max_iterations (default 1000) */
  int32_t method;          /* cfd_ls_method (default CFD_LS_DETECT) */
  int32_t precision;       /* cfd_precision */
  int32_t memory;          /* cfd_memory of b and x */
  int32_t max_outer;       /* FP32_REFINE: refinement steps cap */
  double inner_tolerance;  /* FP32_REFINE: inner relative tolerance */
} cfd_ls_options;
typedef struct {
  int32_t method;       /* cfd_ls_method used (CG or BiCGSTAB) */
  int32_t path;         /* cfd_ls_path */
  int32_t termination;  /* of the Krylov solve (cfd_termination), -1 when none ran */
  int32_t iterations;   /* Krylov iterations */
  double residual;      /* ||D (A x - b)|| / ||D b|| of the returned x */
} cfd_ls_result;
void cfd_ls_options_default(cfd_ls_options* opt);
cfd_status cfd_batch_linear_system_solve(cfd_batch* batch, const cfd_ls_options* opt, const double* b, double* x,
                                         cfd_ls_result* results, cfd_batch_report* rep);
/* Time each pair (threads per system 32..512, systems per CTA 1, 2 or 4) per
 * size bucket on this batch with a fixed iteration budget and keep the fastest
 * (per precision). Several systems per CTA each run on their own named barrier
 * (a warp-wide one for 32-thread systems). */
cfd_status cfd_batch_autotune(cfd_batch* batch, int32_t precision, int32_t sample_iterations);
/* Bucket row limits, chosen threads per system and systems per bucket (4
 * entries each). */
cfd_status cfd_batch_config(const cfd_batch* batch, int32_t precision, int32_t* bucket_rows,
                            int32_t* threads, int32_t* systems);
/* Chosen systems per CTA of the Jacobi-PCG kernel per bucket (4 entries). */
cfd_status cfd_batch_groups(const cfd_batch* batch, int32_t precision, int32_t* groups);
/* Set threads per system (32, 64, 128, 256 or 512) and systems per CTA (1, 2
 * or 4; at most 1024 threads per CTA) per bucket, in place of the autotuner's
 * choice. A bucket whose shared memory does not fit at that choice fails at
 * the next solve with CFD_ERR_CONFIG. */
cfd_status cfd_batch_set_config(cfd_batch* batch, int32_t precision, const int32_t* threads, const int32_t* groups);
cfd_status cfd_batch_destroy(cfd_batch* batch);

/* ---- network assembly on the device --------------------------------------
 * MatrixAssembler::assemble_into (crates/cfd-1d/src/solver/core/
 * matrix_assembly.rs:163-250) for every network of a batch in one launch, so
 * that the Picard loop of NetworkSolver (network_solver.rs:289-340: assemble,
 * then solve from the last iterate) runs without the matrix crossing PCIe.
 * Network s owns global nodes [node_offsets[s], node_offsets[s+1]) and edges
 * [edge_offsets[s], edge_offsets[s+1]); edge_i / edge_j hold node indices
 * LOCAL to the edge's network. fixed[k] != 0 makes global node k a Dirichlet
 * node of pressure fixed_value[k]. The pattern (free-free edges: the 2x2
 * Laplacian block; edges to fixed nodes: the free node's diagonal, eliminated
 * into its right-hand side; fixed nodes: identity rows) is built once here,
 * with duplicate entries of parallel edges summed in edge order. A self-loop
 * is CFD_ERR_CONFIG (:184-189), nodes out of range CFD_ERR_DIM; the per-network
 * limits of cfd_batch_create apply. The batch has no valid matrix until the
 * first cfd_batch_assemble. */
cfd_status cfd_batch_create_networks(cfd_context* ctx, int32_t num_systems, const int64_t* node_offsets,
                                     const int64_t* edge_offsets, const int32_t* edge_i, const int32_t* edge_j,
                                     const int8_t* fixed, const double* fixed_value, cfd_batch** out);
/* Values (FP64 and the FP32 copy) and right-hand sides from per-edge
 * conductances (total-edges entries) and optional Neumann sources (one per
 * node, NULL for none; a fixed node's is ignored), both in `memory`
 * (CFD_MEMORY_HOST or CFD_MEMORY_DEVICE). A non-finite or non-positive
 * conductance is CFD_ERR_CONFIG naming the first such edge (:191-203); a
 * non-finite assembled entry or right-hand side (a source or fixed pressure
 * that is not finite, an overflowing sum) is CFD_ERR_NONFINITE, as
 * validate_linear_system rejects it (solver_detection.rs:66-93). After either
 * the batch holds no valid matrix until a successful assembly. A finite entry
 * beyond the FP32 range assembles (FP64 is exact), and FP32_REFINE solves of
 * the batch return CFD_ERR_NONFINITE until an assembly without one. */
cfd_status cfd_batch_assemble(cfd_batch* batch, const double* conductance, const double* neumann,
                              int32_t memory);
/* Copies the batch's current values (nnz) and right-hand sides (total rows)
 * to host arrays; either may be NULL. */
cfd_status cfd_batch_values(cfd_batch* batch, double* val_host, double* rhs_host);
/* The same assembly on the host, through the same pattern and value code, for
 * checks without a device: *nnz_out receives the entry count, and each
 * non-NULL output (row_ptr: total nodes + 1, col: nnz, val: nnz, rhs: total
 * nodes) is filled; conductance is read only when val or rhs is asked for. */
cfd_status cfd_network_assemble_host(int32_t num_systems, const int64_t* node_offsets,
                                     const int64_t* edge_offsets, const int32_t* edge_i,
                                     const int32_t* edge_j, const int8_t* fixed, const double* fixed_value,
                                     const double* conductance, const double* neumann, int64_t* nnz_out,
                                     int64_t* row_ptr, int32_t* col, double* val, double* rhs);

/* ---- diagnostics --------------------------------------------------------
 * The failure path of the bounded device waits (no reference counterpart):
 * every wait of the bulk-copy SpMV pipelines gives up after a bounded number
 * of tries, flags the context and lets the call return CFD_ERR_TIMEOUT. This
 * runs that wait (the same primitive) on a barrier nothing completes, bounded
 * by `tries`, so the path can be exercised without a fault or a hang. Returns
 * CFD_ERR_TIMEOUT with the wait's message; the context stays usable. */
cfd_status cfd_selftest_wait_timeout(cfd_context* ctx, int32_t tries);

/* ---- residual without device allocation ---------------------------------
 * No counterpart in the reference: an addition for callers that cannot
 * allocate device memory -- a solver embedded in a host application whose
 * memory manager has already reserved the device memory, or a latency-critical
 * loop (a per-time-step convergence monitor, network solves issued from
 * parallel design-search workers) where cudaMalloc/cudaFree would synchronize
 * the device and serialize threads.
 * Computes r = b - A x and *norm2 = ||r||_2^2 (FP64) on device arrays the
 * caller owns: CSR (int32 row_ptr[nrows+1], int32 col[nnz], double val[nnz]),
 * x[ncols], b[nrows], outputs r[nrows] and one double at norm2, enqueued on
 * cuda_stream (NULL: the legacy default stream). It calls no cudaMalloc,
 * cudaFree or allocating library routine: the reduction scratch is a 1 MiB
 * array compiled into the library, held on every GPU that loads it until the
 * process exits. Limit: nrows <= 33 546 240 (one partial sum per 256 rows);
 * larger inputs return CFD_ERR_DIM. The first call on a device looks up the
 * array's device address (set-up) and should come before any stream capture.
 * All calls share the array, so calls that overlap on the GPU (other streams,
 * other threads) race; serialize them. The looked-up address is kept for the
 * life of the process: do not use this entry point on a device after
 * cudaDeviceReset (the library's module, and with it the array, may then sit
 * at another address). */
cfd_status cfd_residual_norm_noalloc(int64_t nrows, int64_t ncols, const int32_t* row_ptr,
                                     const int32_t* col, const double* val, const double* x,
                                     const double* b, double* r, double* norm2, void* cuda_stream);

/* ---- per-kernel statistics of the last solve --------------------------- */
typedef struct {
  int64_t launches;         /* kernels launched by the library in the last cfd_solve */
  int64_t spmv_launches;
  double spmv_bytes;        /* algorithmic bytes moved by SpMV kernels in the last solve */
} cfd_kernel_stats;
cfd_status cfd_last_kernel_stats(cfd_context* ctx, cfd_kernel_stats* out);

#ifdef __cplusplus
}
#endif
#endif /* CFDGPU_H */
