// Device plan of one factored topology: the LU pattern in pivot (internal)
// order plus everything the batched refactor and the four triangular sweeps
// need, as flat int32 arrays ready to upload.
#pragma once
#include <cstdint>
#include <memory>
#include <utility>
#include <vector>

namespace nsg {

// Largest update map a plan carries (int32 words; default 2^30, 4 GiB),
// process-wide (nsg_set_update_map_limit).
int64_t update_map_limit();
void set_update_map_limit(int64_t words);

// An allocator whose resize() leaves new int32 elements uninitialised: the
// refactor's update map (one word per multiply-subtract, gigabytes for large
// grids) is written entirely by the threads that fill it, so each thread
// first-touches its own pages instead of one thread zeroing them all.
template <class T>
struct UninitAllocator : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = UninitAllocator<U>;
    };
    UninitAllocator() = default;
    template <class U>
    UninitAllocator(const UninitAllocator<U>&) noexcept {}
    template <class U>
    void construct(U* p) noexcept {
        ::new (static_cast<void*>(p)) U;
    }
    template <class U, class... Args>
    void construct(U* p, Args&&... args) {
        ::new (static_cast<void*>(p)) U(std::forward<Args>(args)...);
    }
};

class MarkowitzOrder;
class AmdLuFactor;

// Engines whose pivot sequence a plan replays.
enum PlanKindHost : int32_t {
    kPlanKindMarkowitz = 0,  // SparseMatrix (Sparse 1.3): U scaled by 1/pivot
    kPlanKindAmdLu = 1,      // AmdLuSolver: L scaled by 1/pivot
};

struct TopologyPlan {
    int32_t kind = kPlanKindMarkowitz;
    int32_t n = 0;
    int32_t nnz_a = 0;   // slots of the caller's CSC pattern
    int32_t nnz_lu = 0;  // originals + fill-ins
    int32_t max_col = 0; // longest LU column

    // internal index i (0-based) -> external row / column (0-based).
    std::vector<int32_t> perm_row, perm_col;

    // LU in CSC, internal order.  In column j: positions
    // col_ptr[j]..diag_pos[j]-1 are U (rows < j), diag_pos[j] is the pivot,
    // diag_pos[j]+1..col_ptr[j+1]-1 are L (rows > j).  Markowitz plans keep
    // rows ascending; AMD-LU plans keep the U rows in the order the
    // refactor must apply them (the reach's topological order) and the L
    // rows in the reference's stored order.
    std::vector<int32_t> col_ptr, row_idx, diag_pos;

    // Load map: per LU position, the caller's CSC slot, or -1 for a fill-in.
    std::vector<int32_t> lu_src;
    // Inverse: per caller slot, its LU position.
    std::vector<int32_t> a_to_lu;

    // Refactor update map.  For the U entry at position q = (r, j):
    // upd_start[q] indexes upd_dst, where the |L(:, r)| destinations of
    // L(:, r)'s rows are stored in L(:, r)'s order, as positions relative to
    // the start of column j.
    std::vector<int32_t> upd_start;
    std::vector<int32_t, UninitAllocator<int32_t>> upd_dst;
    // False when the map would exceed update_map_limit(): upd_start is then
    // all zero, upd_dst empty, and the grid-wide refactor finds each
    // destination through a per-warp row -> position map instead.
    bool has_update_map = true;

    // L by rows (strictly lower, columns ascending) and U by rows (strictly
    // upper, columns ascending): LU position and column of each entry.
    std::vector<int32_t> lrow_ptr, lrow_pos, lrow_col;
    std::vector<int32_t> urow_ptr, urow_pos, urow_col;
    // Per LU position: its index in the row-major copy of L (rows > column)
    // or of U (rows < column), which the refactor writes alongside the
    // column-major values so the sweeps read contiguous rows; -1 for pivots.
    std::vector<int32_t> rowcopy_pos;
    // Per LU position q of a U entry (r, j): {r, diag_pos[r], |L(:, r)|,
    // upd_start[q]} packed as four int32 (zeros elsewhere), so one 16-byte
    // load gives the refactor everything it needs to apply entry q.
    std::vector<int32_t> umeta;

    // Level schedules (ptr over levels, then members sorted by level).
    //   col:  column j after every r with U(r, j) != 0  (refactor and the
    //         forward sweep of the transposed solve)
    //   fwd:  row i after every c with L(i, c) != 0      (forward solve)
    //   bwd:  row i after every c with U(i, c) != 0      (backward solve)
    //   tbw:  column i after every r with L(r, i) != 0   (transposed backward)
    std::vector<int32_t> col_lev_ptr, col_lev;
    std::vector<int32_t> fwd_lev_ptr, fwd_lev;
    std::vector<int32_t> bwd_lev_ptr, bwd_lev;
    std::vector<int32_t> tbw_lev_ptr, tbw_lev;

    // AMD-LU plans only (empty otherwise), per column k: the pivot's rank
    // among the candidate rows (pivot + L rows, in reach order; -1 when the
    // pivot was outside the reach), and the position, relative to the
    // column start, of the entry that receives diag_gmin (the row of the
    // column's own diagonal element of A), or -1 when the column has none.
    std::vector<int32_t> piv_rank, gmin_pos;

    // Algorithmic work: multiply-subtract updates of one refactor (each is
    // 2 flops), and the reciprocal pivots.
    int64_t updates = 0;

    int64_t refactor_flops() const { return 2 * updates + n; }
    // Compulsory bytes of one refactor: read A, write LU, the index stream
    // (update map + LU pattern), the reciprocal diagonal.
    int64_t refactor_bytes() const {
        return 8LL * nnz_a + 8LL * nnz_lu + (map16() ? 2LL : 4LL) * updates +
               4LL * (nnz_lu + n) + 8LL * n;
    }
    // The device copy of the update map is packed as uint16 positions when
    // every column is short enough for them.
    bool map16() const { return has_update_map && max_col <= 65536; }
    int64_t solve_bytes() const { return 12LL * nnz_lu + 16LL * n; }

    // Total int32 words this plan occupies on the device.
    int64_t device_words() const;
    // Append all arrays to pool; offsets (in int32 words) go to off[].
    void append_to(std::vector<int32_t>& pool, int64_t* off) const;
};

// Build from the host ordering engine after order_and_factor.  slot_elem[k]
// is the engine element of caller CSC slot k.
TopologyPlan build_plan(const MarkowitzOrder& mo, const std::vector<int32_t>& slot_elem);

// Build from the AMD-LU engine after a successful factor(): the pivot
// sequence, L/U structure and replay order of AmdLuSolver::factor_.
TopologyPlan build_plan_amd(const AmdLuFactor& f);

// Build from an exported structure (the reference's own NeoSolver state):
// elements column by column in internal order (1-based rows/cols), the slot
// map and 1-based permutations.  Throws std::invalid_argument on a malformed
// structure.
TopologyPlan build_plan_from_structure(int32_t n, int32_t nnz_a,
                                       const int32_t* int_to_ext_row,
                                       const int32_t* int_to_ext_col,
                                       int32_t n_elem, const int32_t* elem_row,
                                       const int32_t* elem_col,
                                       const int32_t* slot_to_elem);

}  // namespace nsg
