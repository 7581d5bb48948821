// Host-side symbolic phase of the AMD-ordered LU engine.
//
// The reference selects this engine for linear circuits of 256 or more
// unknowns (src/core/make_solver.cpp:156-178): an AMD column ordering on the
// symmetrised pattern, then a left-looking sparse LU with threshold partial
// pivoting whose pivot sequence and fill are fixed afterwards and replayed by
// every later refactorize() (src/core/amd_lu_solver.cpp:11-358).  The GPU
// replays the factorization; this file produces, on the host, exactly the
// ordering and the pivot sequence the reference's AmdLuSolver produces, so
// that the replayed values are bit-identical.
#pragma once
#include <cstdint>
#include <vector>

namespace nsg {

// amd_ordering (src/core/amd.cpp:14-143): exact minimum degree on the
// symmetrised pattern with explicit fill cliques, ties to the lowest index;
// nodes of degree above max(16, 10*sqrt(n)) (capped at n) are set aside and
// appended last by ascending original degree.  perm[k] = original column
// eliminated at step k.  The selection uses a tournament tree over the nodes
// and each clique is formed by sorted merges, so the ordering is the
// reference's at O(log n) per degree change instead of O(n) per step.
std::vector<int32_t> amd_order(int32_t n, const int32_t* col_ptr, const int32_t* row_idx);

// AmdLuSolver's symbolic() + factor_() state.
class AmdLuFactor {
public:
    // AmdLuSolver::symbolic (amd_lu_solver.cpp:11-38): keep the caller's CSC
    // pattern (0-based, rows ascending) and compute the AMD order.
    AmdLuFactor(int32_t n, std::vector<int32_t> col_ptr, std::vector<int32_t> row_idx);

    // AmdLuSolver::factor_ (amd_lu_solver.cpp:74-197): reach of each column
    // in the graph of L by depth-first search, sparse triangular solve in
    // the reach's topological order, threshold partial pivoting (tol 1e-3,
    // diagonal preferred when within tol of the column maximum).  Returns
    // false when the reference reports a singular matrix.
    bool factor(const double* values, double diag_gmin);

    int32_t size() const { return n_; }
    int32_t nnz() const { return static_cast<int32_t>(a_rowidx_.size()); }
    const std::vector<int32_t>& col_ptr() const { return a_colptr_; }
    const std::vector<int32_t>& row_idx() const { return a_rowidx_; }
    // q[k]: original column eliminated at step k.
    const std::vector<int32_t>& q() const { return q_; }
    // pinv[r]: pivot step of original row r.
    const std::vector<int32_t>& pinv() const { return pinv_; }
    // L and U in CSC over pivot steps, as the reference stores them: L(:, k)
    // starts with the unit diagonal, then the sub-diagonal rows in the
    // order the reach listed them; U(:, k) holds the above-diagonal rows in
    // the reach's topological order and ends with the pivot.
    const std::vector<int32_t>& Lp() const { return Lp_; }
    const std::vector<int32_t>& Li() const { return Li_; }
    const std::vector<double>& Lx() const { return Lx_; }
    const std::vector<int32_t>& Up() const { return Up_; }
    const std::vector<int32_t>& Ui() const { return Ui_; }
    const std::vector<double>& Ux() const { return Ux_; }
    // Position of the chosen pivot among the candidate rows of step k (the
    // not-yet-pivotal rows of the reach, in reach order); the candidates
    // other than the pivot are L(:, k)'s rows in stored order.
    const std::vector<int32_t>& piv_rank() const { return piv_rank_; }
    bool factored() const { return factored_; }

private:
    int32_t n_;
    std::vector<int32_t> a_colptr_, a_rowidx_, q_, pinv_;
    std::vector<int32_t> Lp_, Li_, Up_, Ui_, piv_rank_;
    std::vector<double> Lx_, Ux_;
    bool factored_ = false;
};

}  // namespace nsg
