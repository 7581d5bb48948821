/*
 * nsgpu — B200 (sm_100a) batched FP64 sparse refactor and triangular solves
 * for the neospice Newton inner loop, behind a plain C ABI.
 *
 * Conventions
 *   - Every entry point returns an int status: NSG_OK, or an NSG_ERR_* code
 *     with a message available from nsg_last_error() (per thread).  No C++
 *     exception crosses this boundary.
 *   - Pointers named d_* are device pointers (cudaMalloc / torch CUDA
 *     memory) on the current device; `stream` is a cudaStream_t (may be 0).
 *     All other pointers are host memory.
 *   - Matrices are given in the caller's CSC pattern (0-based, rows
 *     ascending within a column), exactly the slot order of the reference's
 *     SparsityPattern / NumericMatrix (src/core/matrix.hpp:16-93).
 *   - Per-instance status codes mirror SparseError (src/solver/error.hpp:5-13):
 *     0 OK, 102 singular (zero pivot), plus 103 when a re-validated pivot
 *     fails the relative threshold and the instance needs a host re-order.
 */
#ifndef NSGPU_H
#define NSGPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define NSG_OK 0
#define NSG_ERR_INVALID 1    /* bad argument or misuse (reference: std::logic_error / invalid_argument) */
#define NSG_ERR_CUDA 2       /* a CUDA runtime call failed */
#define NSG_ERR_NOMEM 8      /* SparseError::NoMemory */
#define NSG_SINGULAR 102     /* SparseError::Singular / ZeroDiag */
#define NSG_REORDER 103      /* pivot failed re-validation: run nsg_topology_numeric */

typedef struct nsg_topology nsg_topology;
typedef struct nsg_batch nsg_batch;

/* Message of the last failing call on this thread ("" if none). */
const char* nsg_last_error(void);

/* ---- Symbolic phase (host) ------------------------------------------------
 * nsg_topology_order: NeoSolver::symbolic followed by the first
 * NeoSolver::numeric (src/core/neo_solver.cpp:184-245): load values, MNA
 * pre-order, add diag_gmin, Markowitz order_and_factor with relThr 1e-3,
 * absThr 1e-13 and diagonal pivoting (src/solver/factor.cpp:911-978).  The
 * pivot sequence and fill pattern are bit-identical to the reference's.
 * Returns NSG_SINGULAR (and no topology) when the reference would report a
 * singular matrix. */
int nsg_topology_order(int n, int nnz, const int* col_ptr, const int* row_idx,
                       const double* values, double diag_gmin, nsg_topology** out);

/* nsg_topology_numeric: a later NeoSolver::numeric on the same topology
 * (neo_solver.cpp:219-245): re-validate every pivot on the new values and
 * re-order from the first failing step, as SparseMatrix::order_and_factor
 * does (factor.cpp:929-947).  *reordered is set to the first re-ordered step
 * (1-based) or 0.  Instances sharing this topology in an existing batch must
 * be rebuilt when *reordered != 0. */
int nsg_topology_numeric(nsg_topology* topo, const double* values, double diag_gmin,
                         int* reordered);

/* nsg_topology_import: take a symbolic result computed by the reference's
 * own NeoSolver (the state behind element_ptrs_ after order_and_factor,
 * neo_solver.cpp:113-146): 1-based int_to_ext_row/col of length n, n_elem
 * elements listed column by column in pivot order with 1-based internal
 * rows (ascending) and columns, and for each of the nnz caller slots its
 * element index. */
int nsg_topology_import(int n, int nnz, const int* int_to_ext_row,
                        const int* int_to_ext_col, int n_elem, const int* elem_row,
                        const int* elem_col, const int* slot_to_elem, nsg_topology** out);

/* Sizes: n, caller nnz, LU entries, multiply-subtract updates per refactor,
 * and the level counts of the refactor / forward / backward schedules. */
int nsg_topology_info(const nsg_topology* topo, int* n, int* nnz, int* nnz_lu,
                      long long* updates, int* col_levels, int* fwd_levels,
                      int* bwd_levels);

/* Export in the format nsg_topology_import takes (arrays sized n, n, nnz_lu,
 * nnz_lu, nnz). */
int nsg_topology_export(const nsg_topology* topo, int* int_to_ext_row,
                        int* int_to_ext_col, int* elem_row, int* elem_col,
                        int* slot_to_elem);

void nsg_topology_free(nsg_topology* topo);

/* ---- Batches (device) -----------------------------------------------------
 * A batch holds `count` instances, instance i using topos[i] (instances may
 * share a topology).  It owns the device plan and the LU values.  The
 * caller's value and vector arrays are packed instance after instance; the
 * offsets (count+1 entries each, in doubles) come from nsg_batch_layout. */
int nsg_batch_create(int count, nsg_topology* const* topos, nsg_batch** out);
void nsg_batch_free(nsg_batch* batch);
int nsg_batch_layout(const nsg_batch* batch, long long* value_offsets,
                     long long* vector_offsets, long long* lu_offsets);

/* spFactor for every instance: SparseMatrix::factor after load_real and
 * add_diag_gmin (neo_solver.cpp:247-265, factor.cpp:980-1052), with the
 * fixed pivots.  check_pivots != 0 instead applies the re-validation test of
 * a later NeoSolver::numeric (factor.cpp:929-947) and reports NSG_REORDER.
 * d_status[i] / d_fail_step[i] (device int arrays, fail_step optional)
 * receive the per-instance code and the failing 0-based pivot step. */
int nsg_batch_refactor(nsg_batch* batch, const double* d_values, double diag_gmin,
                       int check_pivots, int* d_status, int* d_fail_step, void* stream);

/* spSolve: d_x holds b on entry and x on return, per instance
 * (SparseMatrix::solve, src/solver/solve.cpp:6-47; NeoSolver::solve). */
int nsg_batch_solve(nsg_batch* batch, double* d_x, void* stream);

/* spSolveTransposed: A^T x = b on the same factors
 * (SparseMatrix::solve_transposed, src/solver/solve.cpp:102-141). */
int nsg_batch_solve_transposed(nsg_batch* batch, double* d_x, void* stream);

/* Device pointer to the factored LU values (layout per nsg_batch_layout and
 * the topology export: L unscaled, U scaled by the reciprocal pivot, pivots
 * stored as reciprocals — the reference's in-place element values). */
const double* nsg_batch_lu(const nsg_batch* batch);

/* Synchronous copy of all LU values to host memory (lu_offsets[count]
 * doubles). */
int nsg_batch_lu_to_host(const nsg_batch* batch, double* out);

#ifdef __cplusplus
}
#endif

#endif /* NSGPU_H */
