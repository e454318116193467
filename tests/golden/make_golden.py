"""Writes tests/golden/reference_golden.json: the known-answer vectors of the
CFDrs unit tests for this path, transcribed from the reference's test sources
(paths relative to the CFDrs repository). The reference is Rust and cannot be
built here, so these vectors -- not a run of the reference -- pin the oracle.

Run: python tests/golden/make_golden.py
"""
import json
import os

GOLDEN = {
    "smoother_tridiagonal_5": {
        "source": "crates/cfd-math/src/linear_solver/preconditioners/multigrid/smoothers.rs:395-492",
        "matrix": "5x5 tridiagonal [-1, 2, -1]",
        "b": [1.0, 2.0, 3.0, 4.0, 5.0],
        "x0": [0.0, 0.0, 0.0, 0.0, 0.0],
        "relaxation": 1.0,
        "sweeps": 1,
        "jacobi": [0.5, 1.0, 1.5, 2.0, 2.5],
        "gauss_seidel": [0.5, 1.25, 2.125, 3.0625, 4.03125],
        "symmetric_gauss_seidel": [2.291015625, 3.58203125, 4.6640625, 5.078125, 4.03125],
        "sor_1": [0.5, 1.25, 2.125, 3.0625, 4.03125],
    },
    "strength_grid_4x4": {
        "source": "crates/cfd-math/src/linear_solver/preconditioners/multigrid/coarsening/mod.rs:30-66,108-122",
        "matrix": "4x4 grid Laplacian, 4 on the diagonal, -1 to grid neighbours, row-major",
        "theta": 0.5,
        "nnz": 48,
        "row0_cols": [1, 4],
        "row0_vals": [1.0, 1.0],
        "row5_cols": [1, 4, 6, 9],
        "row5_vals": [1.0, 1.0, 1.0, 1.0],
    },
    "spmv_3x3": {
        "source": "crates/cfd-math/src/sparse/tests.rs:195-221",
        "row_ptr": [0, 2, 3, 5],
        "col": [0, 2, 1, 0, 2],
        "val": [2.0, 1.0, 3.0, 1.0, 2.0],
        "x": [1.0, 2.0, 3.0],
        "y": [5.0, 6.0, 7.0],
        "tol": 1e-10,
    },
    "coarsest_solve_3x3": {
        "source": "crates/cfd-math/src/linear_solver/preconditioners/multigrid/cycles.rs:513-534",
        "row_ptr": [0, 2, 4, 5],
        "col": [0, 1, 1, 2, 2],
        "val": [1.0, 1.0, 1.0, 1.0, 1.0],
        "b": [1.0, 2.0, 3.0],
        "x": [2.0, -1.0, 3.0],
        "tol": 1e-12,
    },
    "diagonal_solve_2": {
        "source": "crates/cfd-math/src/linear_solver/krylov.rs:466-492",
        "row_ptr": [0, 1, 2],
        "col": [0, 1],
        "val": [2.0, 3.0],
        "b": [2.0, 6.0],
        "x": [1.0, 2.0],
        "tolerance": 1e-12,
        "max_iterations": 20,
        "tol": 1e-10,
    },
    "jacobi_tiny_diagonal": {
        "source": "crates/cfd-1d/src/solver/core/linear_system.rs:339-349",
        "row_ptr": [0, 1, 2],
        "col": [0, 1],
        "val": [1.0e-18, 2.0],
        "inv_diag": [1.0, 0.5],
        "tol": 1e-12,
    },
    "amg_poisson_2d_16": {
        "source": "crates/cfd-math/tests/amg_integration_test.rs:17-122,212-268",
        "matrix": "poisson_2d(16): 4 on the diagonal, -1 to grid neighbours",
        "n": 16,
        "manufactured": "x*_k = sin(pi t) + 0.5 t, t = k / n^2; b = A x*",
        "tolerance": 1e-10,
        "max_iterations": 200,
        "max_abs_error": 1e-6,
        "contraction_sizes": [8, 16],
        "contraction_steps": 5,
        "contraction_bound": 1.0,
    },
    "gmres_restart_ladder": {
        "source": "crates/cfd-math/src/linear_solver/krylov.rs:440-463 (RestartWidth::covering, :96-120)",
        "requested_width": [[1, 8], [8, 8], [9, 16], [30, 32], [100, 128], [200, 256], [10000, 256]],
    },
    "gmres_diagonal_2": {
        "source": "crates/cfd-math/src/linear_solver/krylov.rs:466-492 (workspace reused for two solves)",
        "row_ptr": [0, 1, 2],
        "col": [0, 1],
        "val": [2.0, 3.0],
        "b": [2.0, 6.0],
        "x": [1.0, 2.0],
        "restart": 30,
        "tolerance": 1e-12,
        "max_iterations": 20,
        "tol": 1e-10,
    },
    "gmres_basic_5": {
        "source": "crates/cfd-math/tests/simple_gmres_tests.rs:61-93",
        "entries": [[0, 0, 2.0], [0, 1, -1.0], [1, 0, -1.0], [1, 1, 2.0], [1, 2, -1.0], [2, 1, -1.0],
                    [2, 2, 3.0], [2, 3, -1.0], [3, 2, -1.0], [3, 3, 2.0], [3, 4, -1.0], [4, 3, -1.0],
                    [4, 4, 2.0]],
        "n": 5,
        "b": [1.0, 2.0, 3.0, 2.0, 1.0],
        "restart": 4,
        "tolerance": 1e-8,
        "max_iterations": 100,
        "residual_below": 1.5,
    },
    "gmres_restart_8": {
        "source": "crates/cfd-math/tests/simple_gmres_tests.rs:96-121",
        "matrix": "tridiagonal n = 8: 2 on the diagonal, -1 off it; b = 1",
        "n": 8,
        "restart": 3,
        "tolerance": 1e-8,
        "max_iterations": 200,
        "residual_below": 1e-6,
    },
    "gmres_diag_precond_6": {
        "source": "crates/cfd-math/tests/simple_gmres_tests.rs:124-145",
        "matrix": "diagonal 1 + 0.1 i, i < 6; b = 1; identity preconditioner",
        "n": 6,
        "restart": 6,
        "tolerance": 1e-10,
        "max_iterations": 50,
        "residual_below": 1e-8,
    },
    "gmres_core_tridiag_6": {
        "source": "crates/cfd-math/tests/core_solver_tests.rs:125-150",
        "matrix": "tridiagonal n = 6: 3 on the diagonal, -1 off it; b = 1",
        "n": 6,
        "restart": 4,
        "tolerance": 1e-8,
        "max_iterations": 50,
        "residual_below": 0.3,
    },
    "amg_gmres_2d_16": {
        "source": "crates/cfd-math/tests/amg_integration_test.rs:125-142",
        "matrix": "poisson_2d(16), manufactured x*, AMGConfig::default",
        "n": 16,
        "restart": 30,
        "tolerance": 1e-10,
        "max_iterations": 200,
        "max_abs_error": 1e-6,
    },
    "kirchhoff_abc": {
        "source": "crates/cfd-1d/src/solver/core/matrix_assembly.rs:270-410",
        "edges": [[0, 1, 1.0], [1, 2, 2.0]],
        "dirichlet": {"0": 100.0, "2": 0.0},
        "diag_b": 3.0,
        "rhs_b": 100.0,
        "rhs_b_with_neumann_5": 105.0,
        "tol": 1e-12,
    },
    "simple_apply": {
        "source": "crates/cfd-math/src/linear_solver/block_preconditioner.rs:987-1016, 1059-1085",
        "n_velocity": 2,
        "b": [4.0, 4.0, 2.0, 2.0],
        # entries (row, col, value) as the tests' SparseMatrixBuilder adds them
        "stabilized": {"entries": [[0, 0, 4.0], [1, 1, 4.0], [0, 2, 1.0], [1, 3, 1.0], [2, 0, 1.0], [3, 1, 1.0],
                                   [2, 2, 1.0], [3, 3, 1.0]],
                       "x": [0.6666666666666666, 0.6666666666666666, 1.3333333333333333, 1.3333333333333333]},
        "normalized": {"entries": [[0, 0, 4.0], [1, 1, 4.0], [0, 2, -1.0], [1, 3, -1.0], [2, 0, -1.0],
                                   [3, 1, -1.0]],
                       "x": [-2.0, -2.0, -12.0, -12.0]},
        # BlockDiagonalPreconditioner on the stabilized matrix (:1044-1058)
        "block_diagonal": {"b": [4.0, 4.0, 1.0, 1.0], "x": [1.0, 1.0, 1.0, 1.0]},
        "tol": 1e-10,
    },
    "component_block": {
        "source": "crates/cfd-math/src/linear_solver/block_preconditioner.rs:1024-1036, 1100-1116",
        "n_velocity": 6,
        # three velocity components of two rows, 4 on the diagonal; gradient and
        # divergence -1 between u0/p0 and u1/p1; no pressure block
        "entries": [[0, 0, 4.0], [1, 1, 4.0], [2, 2, 4.0], [3, 3, 4.0], [4, 4, 4.0], [5, 5, 4.0],
                    [0, 6, -1.0], [1, 7, -1.0], [6, 0, -1.0], [7, 1, -1.0]],
        "b": [4.0, 4.0, 0.0, 0.0, 0.0, 0.0, 2.0, 2.0],
        "x": [-2.0, -2.0, 0.0, 0.0, 0.0, 0.0, -12.0, -12.0],
        "tol": 1e-10,
    },
    # The reference test checks only that the free block is symmetric; the
    # entries below follow from assemble_into's rules (:208-246) by hand:
    # B = 1 (AB, A fixed) + 3 (BC); C = 2 (AC, A fixed) + 3 (BC) + 4 (CD, D fixed);
    # B-C = -3; RHS_B = 1 * 100, RHS_C = 2 * 100 + 4 * 0.
    "kirchhoff_active_block": {
        "source": "crates/cfd-1d/src/solver/core/matrix_assembly.rs:404-450 (entries derived from :208-246)",
        "edges": [[0, 1, 1.0], [0, 2, 2.0], [1, 2, 3.0], [2, 3, 4.0]],
        "dirichlet": {"0": 100.0, "3": 0.0},
        "dense": [[1.0, 0.0, 0.0, 0.0], [0.0, 4.0, -3.0, 0.0], [0.0, -3.0, 9.0, 0.0], [0.0, 0.0, 0.0, 1.0]],
        "rhs": [100.0, 100.0, 200.0, 0.0],
    },
}


def main():
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_golden.json")
    with open(out, "w") as f:
        json.dump(GOLDEN, f, indent=1, sort_keys=True)
    print(out)


if __name__ == "__main__":
    main()
