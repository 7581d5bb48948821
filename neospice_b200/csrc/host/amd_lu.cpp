#include "amd_lu.hpp"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <utility>

namespace nsg {

namespace {

// Minimum of (degree, index) over the live nodes, as one 64-bit key per leaf
// of a complete binary tree: the root is the node the reference's linear
// scan `degree[i] < best_deg` (src/core/amd.cpp:94-101) would pick.
class MinDegreeTree {
public:
    explicit MinDegreeTree(int32_t n) {
        size_ = 1;
        while (size_ < n) size_ <<= 1;
        key_.assign(2 * static_cast<size_t>(size_), kNone);
    }
    void set(int32_t i, int32_t degree) { put(i, (static_cast<uint64_t>(degree) << 32) | uint32_t(i)); }
    void remove(int32_t i) { put(i, kNone); }
    int32_t top() const { return static_cast<int32_t>(key_[1] & 0xffffffffu); }
    void build() {
        for (int64_t k = size_ - 1; k >= 1; --k) key_[k] = std::min(key_[2 * k], key_[2 * k + 1]);
    }
    void init(int32_t i, int32_t degree) {
        key_[size_ + i] = (static_cast<uint64_t>(degree) << 32) | uint32_t(i);
    }

private:
    static constexpr uint64_t kNone = std::numeric_limits<uint64_t>::max();
    int64_t size_;
    std::vector<uint64_t> key_;
    void put(int32_t i, uint64_t v) {
        int64_t k = size_ + i;
        key_[k] = v;
        for (k >>= 1; k >= 1; k >>= 1) {
            const uint64_t m = std::min(key_[2 * k], key_[2 * k + 1]);
            if (key_[k] == m) break;
            key_[k] = m;
        }
    }
};

}  // namespace

std::vector<int32_t> amd_order(int32_t n, const int32_t* col_ptr, const int32_t* row_idx) {
    if (n <= 0) return {};
    // Symmetrised adjacency without self loops (amd.cpp:20-35).
    std::vector<std::vector<int32_t>> adj(n);
    for (int32_t j = 0; j < n; ++j)
        for (int32_t p = col_ptr[j]; p < col_ptr[j + 1]; ++p) {
            const int32_t i = row_idx[p];
            if (i < 0 || i >= n) throw std::invalid_argument("amd_order: row index out of range");
            if (i != j) {
                adj[j].push_back(i);
                adj[i].push_back(j);
            }
        }
    std::vector<int32_t> degree(n);
    for (int32_t i = 0; i < n; ++i) {
        auto& a = adj[i];
        std::sort(a.begin(), a.end());
        a.erase(std::unique(a.begin(), a.end()), a.end());
        degree[i] = static_cast<int32_t>(a.size());
    }

    // Dense nodes (amd.cpp:37-79): degree above max(16, 10*sqrt(n)), at most n.
    int32_t dense_thresh = static_cast<int32_t>(10.0 * std::sqrt(static_cast<double>(n)));
    dense_thresh = std::max<int32_t>(dense_thresh, 16);
    dense_thresh = std::min<int32_t>(dense_thresh, n);
    std::vector<char> gone(n, 0);
    std::vector<int32_t> dense_nodes;
    for (int32_t i = 0; i < n; ++i)
        if (degree[i] > dense_thresh) {
            gone[i] = 1;
            dense_nodes.push_back(i);
        }
    if (!dense_nodes.empty()) {
        for (int32_t i = 0; i < n; ++i) {
            if (gone[i]) continue;
            auto& a = adj[i];
            a.erase(std::remove_if(a.begin(), a.end(), [&](int32_t v) { return gone[v] != 0; }),
                    a.end());
            degree[i] = static_cast<int32_t>(a.size());
        }
    }

    MinDegreeTree tree(n);
    for (int32_t i = 0; i < n; ++i)
        if (!gone[i]) tree.init(i, degree[i]);
    tree.build();

    std::vector<int32_t> perm;
    perm.reserve(n);
    std::vector<int32_t> nbrs, merged;
    const int32_t steps = n - static_cast<int32_t>(dense_nodes.size());
    for (int32_t step = 0; step < steps; ++step) {
        const int32_t best = tree.top();
        perm.push_back(best);
        gone[best] = 1;
        tree.remove(best);
        nbrs.clear();
        for (int32_t v : adj[best])
            if (!gone[v]) nbrs.push_back(v);  // sorted: adj lists stay sorted
        // The live neighbours become a clique (amd.cpp:111-123) and lose
        // `best` (amd.cpp:125-131): each neighbour's list is merged with the
        // clique, both sorted, dropping itself and eliminated nodes.
        for (int32_t u : nbrs) {
            const auto& a = adj[u];
            merged.clear();
            merged.reserve(a.size() + nbrs.size());
            size_t x = 0, y = 0;
            while (x < a.size() || y < nbrs.size()) {
                int32_t v;
                if (y == nbrs.size() || (x < a.size() && a[x] < nbrs[y])) {
                    v = a[x++];
                } else if (x == a.size() || nbrs[y] < a[x]) {
                    v = nbrs[y++];
                } else {
                    v = a[x++];
                    ++y;
                }
                if (v == u || gone[v]) continue;
                merged.push_back(v);
            }
            adj[u].swap(merged);
            degree[u] = static_cast<int32_t>(adj[u].size());
            tree.set(u, degree[u]);
        }
        std::vector<int32_t>().swap(adj[best]);
    }

    // Dense nodes last, by ascending original degree (amd.cpp:134-142); the
    // same std::sort call on the same sequence gives the same order.
    std::sort(dense_nodes.begin(), dense_nodes.end(),
              [&](int32_t a, int32_t b) { return degree[a] < degree[b]; });
    for (int32_t d : dense_nodes) perm.push_back(d);
    return perm;
}

AmdLuFactor::AmdLuFactor(int32_t n, std::vector<int32_t> col_ptr, std::vector<int32_t> row_idx)
    : n_(n), a_colptr_(std::move(col_ptr)), a_rowidx_(std::move(row_idx)) {
    if (n_ <= 0 || static_cast<int32_t>(a_colptr_.size()) != n_ + 1)
        throw std::invalid_argument("AmdLuFactor: bad pattern");
    q_ = amd_order(n_, a_colptr_.data(), a_rowidx_.data());
    if (static_cast<int32_t>(q_.size()) != n_) {
        q_.resize(n_);
        for (int32_t i = 0; i < n_; ++i) q_[i] = i;
    }
    pinv_.assign(n_, -1);
}

bool AmdLuFactor::factor(const double* values, double diag_gmin) {
    constexpr double kPivotTol = 1e-3;  // AmdLuSolver::pivot_tol_
    const int32_t n = n_;
    factored_ = false;
    Lp_.assign(n + 1, 0);
    Up_.assign(n + 1, 0);
    Li_.clear();
    Lx_.clear();
    Ui_.clear();
    Ux_.clear();
    piv_rank_.assign(n, 0);
    pinv_.assign(n, -1);
    std::vector<double> x(n, 0.0);
    std::vector<int32_t> xi(n), path(n), resume(n);
    std::vector<char> seen(n, 0);

    // Depth-first search from `start` over the graph of the L columns
    // computed so far (row r leads to the rows of L(:, pinv[r])); finished
    // nodes are written to xi[--top], so xi[top..n) is a topological order.
    auto reach = [&](int32_t start, int32_t top) {
        int32_t depth = 0;
        path[0] = start;
        while (depth >= 0) {
            const int32_t r = path[depth];
            const int32_t col = pinv_[r];
            if (!seen[r]) {
                seen[r] = 1;
                resume[depth] = col < 0 ? 0 : Lp_[col];
            }
            const int32_t end = col < 0 ? 0 : Lp_[col + 1];
            bool descended = false;
            for (int32_t p = resume[depth]; p < end; ++p) {
                const int32_t i = Li_[p];
                if (seen[i]) continue;
                resume[depth] = p;
                path[++depth] = i;
                descended = true;
                break;
            }
            if (!descended) {
                --depth;
                xi[--top] = r;
            }
        }
        return top;
    };

    for (int32_t k = 0; k < n; ++k) {
        const int32_t col = q_[k];
        Lp_[k] = static_cast<int32_t>(Li_.size());
        Up_[k] = static_cast<int32_t>(Ui_.size());
        int32_t top = n;
        for (int32_t p = a_colptr_[col]; p < a_colptr_[col + 1]; ++p)
            if (!seen[a_rowidx_[p]]) top = reach(a_rowidx_[p], top);
        for (int32_t p = top; p < n; ++p) x[xi[p]] = 0.0;
        for (int32_t p = a_colptr_[col]; p < a_colptr_[col + 1]; ++p) x[a_rowidx_[p]] = values[p];
        if (diag_gmin != 0.0) x[col] += diag_gmin;

        // x = L \ A(:, col) over the reach, in topological order.
        for (int32_t px = top; px < n; ++px) {
            const int32_t j = xi[px];
            const int32_t J = pinv_[j];
            if (J < 0) continue;
            const double xj = x[j];
            for (int32_t p = Lp_[J] + 1; p < Lp_[J + 1]; ++p) x[Li_[p]] -= Lx_[p] * xj;
        }

        // Threshold partial pivoting among the rows not yet pivotal.
        int32_t ipiv = -1;
        double amax = -1.0;
        for (int32_t p = top; p < n; ++p) {
            const int32_t i = xi[p];
            if (pinv_[i] < 0) {
                const double t = std::fabs(x[i]);
                if (t > amax) {
                    amax = t;
                    ipiv = i;
                }
            } else {
                Ui_.push_back(pinv_[i]);
                Ux_.push_back(x[i]);
            }
        }
        auto unmark = [&]() {
            for (int32_t p = top; p < n; ++p) seen[xi[p]] = 0;
        };
        if (ipiv == -1 || amax <= 0.0) {
            unmark();
            return false;
        }
        if (pinv_[col] < 0 && std::fabs(x[col]) >= amax * kPivotTol) ipiv = col;
        const double pivot = x[ipiv];
        if (pivot == 0.0) {
            unmark();
            return false;
        }
        Ui_.push_back(k);
        Ux_.push_back(pivot);
        pinv_[ipiv] = k;
        Li_.push_back(ipiv);
        Lx_.push_back(1.0);
        // -1: the pivot row was not in the reach (only possible through
        // diag_gmin on a structurally absent diagonal).
        piv_rank_[k] = -1;
        for (int32_t p = top; p < n; ++p) {
            const int32_t i = xi[p];
            if (i == ipiv) piv_rank_[k] = static_cast<int32_t>(Li_.size()) - Lp_[k] - 1;
            if (pinv_[i] < 0) {
                Li_.push_back(i);
                Lx_.push_back(x[i] / pivot);
            }
            x[i] = 0.0;
        }
        unmark();
    }
    Lp_[n] = static_cast<int32_t>(Li_.size());
    Up_[n] = static_cast<int32_t>(Ui_.size());
    for (auto& r : Li_) r = pinv_[r];
    factored_ = true;
    return true;
}

}  // namespace nsg
