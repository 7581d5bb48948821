// Device-side descriptors shared by the host batch code and the kernels.
#pragma once
#include <cstdint>

namespace nsg {

// Index of each plan array in PlanDesc::off; order matches the host's
// NSG_PLAN_ARRAYS list in plan.cpp.
enum PlanArray : int {
    PA_perm_row, PA_perm_col, PA_col_ptr, PA_row_idx, PA_diag_pos, PA_lu_src,
    PA_upd_start, PA_upd_dst, PA_lrow_ptr, PA_lrow_pos, PA_lrow_col, PA_urow_ptr,
    PA_urow_pos, PA_urow_col, PA_col_lev_ptr, PA_col_lev, PA_fwd_lev_ptr, PA_fwd_lev,
    PA_bwd_lev_ptr, PA_bwd_lev, PA_tbw_lev_ptr, PA_tbw_lev, PA_rowcopy_pos, PA_umeta,
    PA_piv_rank, PA_gmin_pos, PA_COUNT
};

struct PlanDesc {
    int32_t n, nnz_a, nnz_lu;
    int32_t n_col_lev, n_fwd_lev, n_bwd_lev, n_tbw_lev;
    int32_t max_col;  // longest LU column
    int32_t nnz_l, nnz_u;  // strictly lower / upper entries
    int32_t kind;          // kPlanMarkowitz or kPlanAmdLu
    int32_t has_map;       // 1: PA_upd_start / PA_upd_dst hold the update map
    int32_t map16;         // 1: the update map is packed as uint16 positions
                           // (every column is shorter than 65,537 rows)
    int64_t off[PA_COUNT];  // int32-word offsets into the plan pool
    int64_t words;          // words from off[0] that hold all of the plan's arrays
};

#ifdef __CUDACC__
// Entry k of a plan's update map: the position in column j that update k
// of U(r, j) writes.  Packed plans (map16) hold it in 16 bits, halving the
// map reads of the refactor; the values are the same.
__device__ __forceinline__ int32_t upd_at(const int32_t* upd_dst, int32_t map16, int64_t k) {
    return map16 ? static_cast<int32_t>(reinterpret_cast<const uint16_t*>(upd_dst)[k])
                 : upd_dst[k];
}
#endif

struct InstDesc {
    int32_t plan;   // index into the PlanDesc array
    int32_t index;  // the instance's position in the caller's arrays
    int64_t a_off;   // into the caller's A values (doubles)
    int64_t lu_off;  // into the batch's LU values
    int64_t x_off;   // into the caller's rhs / solution vectors
    int64_t w_off;   // into the batch's sweep workspace
    int64_t lrows_off;  // into the batch's row-major L copy
    int64_t urows_off;  // into the batch's row-major U copy
};

// Engine whose factorization a plan replays.
//   kPlanMarkowitz: SparseMatrix::factor (src/solver/factor.cpp:980-1052).
//     U(r, j) = a(r, j) * (1 / p_r), L unscaled, the pivot stored as its
//     reciprocal; U entries applied in ascending row order.
//   kPlanAmdLu: AmdLuSolver::refactor_replay_ (src/core/amd_lu_solver.cpp:
//     214-271).  U unscaled, L(i, k) = x_i / u_kk, the pivot stored as is; U
//     entries applied in the stored (reach) order.
enum : int32_t { kPlanMarkowitz = 0, kPlanAmdLu = 1 };

// What a refactor checks beyond an exact zero pivot.
//   kCheckNone:     nothing (spFactor; a replay whose pivots the host chose).
//   kCheckNumeric:  a numeric() on an already factored solver.  Markowitz:
//     the pivot re-validation of order_and_factor (factor.cpp:929-947).
//     AMD-LU: factor_'s threshold pivot choice (amd_lu_solver.cpp:134-157)
//     must pick the plan's pivot row.  Failure -> kStatusReorder.
//   kCheckRefactor: a refactorize().  Markowitz: as kCheckNone.  AMD-LU: the
//     replay's pivot-growth test (amd_lu_solver.cpp:256-259); failure ->
//     kStatusReorder (the reference falls back to a full factor_).
enum : int { kCheckNone = 0, kCheckNumeric = 1, kCheckRefactor = 2 };

// Per-instance status codes written by the refactor.
enum : int32_t {
    kStatusOk = 0,
    kStatusSingular = 102,  // exact zero pivot (SparseError::ZeroDiag)
    kStatusReorder = 103,   // pivot failed the relative threshold
    kStatusTimeout = 104,   // a bounded dependency wait gave up (no result)
    kStatusNeedOrder = 105, // a solver's first numeric(): the host orders on this matrix
};

}  // namespace nsg
