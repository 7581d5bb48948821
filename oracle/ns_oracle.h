/*
 * Test infrastructure only (the oracle): a plain-C restatement of the
 * reference's fixed-pivot refactor and triangular solves, used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker.
 * The product never links it.
 *
 * Structure arguments use the export format of the reference's NeoSolver
 * state (oracle/ref_shim.cpp, nsref_solver_export): n_elem elements listed
 * column by column in internal (pivot) order, 1-based internal rows
 * ascending within a column, 1-based internal columns; slot_to_elem maps the
 * caller's nnz CSC slots to elements; int_to_ext_row/col are 1-based.
 */
#ifndef NS_ORACLE_H
#define NS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Load A, add diag_gmin to the pivots and refactor with fixed pivots.
 * check_pivots = 0: SparseMatrix::factor (src/solver/factor.cpp:980-1052),
 *   returns 102 at the first exact zero pivot.
 * check_pivots = 1: the re-validation loop of SparseMatrix::order_and_factor
 *   (factor.cpp:929-947), returns 103 at the first pivot not above 1e-3 x the
 *   largest entry below it.
 * *fail_step receives the failing 0-based step (or -1).  lu has n_elem
 * entries. */
int nso_refactor(int n, int nnz, int n_elem, const int* elem_row, const int* elem_col,
                 const int* slot_to_elem, const double* a, double diag_gmin,
                 int check_pivots, double* lu, int* fail_step);

/* SparseMatrix::solve (src/solver/solve.cpp:6-47): x holds b on entry. */
int nso_solve(int n, int n_elem, const int* elem_row, const int* elem_col,
              const int* int_to_ext_row, const int* int_to_ext_col, const double* lu,
              double* x);

/* SparseMatrix::solve_transposed (src/solver/solve.cpp:102-141). */
int nso_solve_transposed(int n, int n_elem, const int* elem_row, const int* elem_col,
                         const int* int_to_ext_row, const int* int_to_ext_col,
                         const double* lu, double* x);

#ifdef __cplusplus
}
#endif

#endif
