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

/* ---- AMD-LU (src/core/amd_lu_solver.cpp) ------------------------------------
 * Factor arguments use AmdLuSolver's own storage (oracle/ref_shim.cpp,
 * nsref_amdlu_export): q[k] the column of step k, pinv[r] the step of row r,
 * L in CSC over steps with the unit diagonal first (Lp, Li), U in CSC over
 * steps with the pivot last (Up, Ui); a_colptr/a_rowidx the caller's CSC. */

/* AmdLuSolver::refactor_replay_ (amd_lu_solver.cpp:214-271) on values a:
 * writes Lx and Ux.  Returns 0 on success, 103 when the pivot-growth test
 * fails at a step (*fail_step receives it; the reference would re-factor). */
int nso_amd_replay(int n, const int* a_colptr, const int* a_rowidx, const int* q,
                   const int* pinv, const int* Lp, const int* Li, const int* Up, const int* Ui,
                   const double* a, double diag_gmin, double* Lx, double* Ux, int* fail_step);

/* AmdLuSolver::solve (amd_lu_solver.cpp:303-344): x holds b on entry. */
int nso_amd_solve(int n, const int* q, const int* pinv, const int* Lp, const int* Li,
                  const double* Lx, const int* Up, const int* Ui, const double* Ux, double* x);

#ifdef __cplusplus
}
#endif

#endif
