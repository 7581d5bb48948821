#include "plan.hpp"

#include "amd_lu.hpp"
#include "sparse_order.hpp"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <string>
#include <thread>

namespace nsg {

namespace {
std::atomic<int64_t> g_update_map_limit{int64_t{1} << 30};
}  // namespace

int64_t update_map_limit() { return g_update_map_limit.load(); }
void set_update_map_limit(int64_t words) { g_update_map_limit.store(words); }

namespace {

// Counting sort of items by level; returns (ptr over levels, members).
void level_sort(const std::vector<int32_t>& level, std::vector<int32_t>& ptr,
                std::vector<int32_t>& members) {
    int32_t nlev = 0;
    for (int32_t l : level) nlev = std::max(nlev, l + 1);
    ptr.assign(nlev + 1, 0);
    for (int32_t l : level) ++ptr[l + 1];
    for (int32_t l = 0; l < nlev; ++l) ptr[l + 1] += ptr[l];
    members.assign(level.size(), 0);
    std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
    for (int32_t i = 0; i < static_cast<int32_t>(level.size()); ++i)
        members[fill[level[i]]++] = i;
}

// Derive everything from the CSC LU pattern (col_ptr/row_idx/lu_src set).
void finish(TopologyPlan& p) {
    const int32_t n = p.n;
    p.nnz_lu = static_cast<int32_t>(p.row_idx.size());
    p.diag_pos.assign(n, -1);
    for (int32_t j = 0; j < n; ++j) {
        for (int32_t q = p.col_ptr[j]; q < p.col_ptr[j + 1]; ++q) {
            if (p.kind == kPlanKindMarkowitz && q > p.col_ptr[j] &&
                p.row_idx[q] <= p.row_idx[q - 1])
                throw std::invalid_argument("plan: rows not ascending in column " +
                                            std::to_string(j));
            if (p.row_idx[q] == j) p.diag_pos[j] = q;
        }
        if (p.diag_pos[j] < 0)
            throw std::invalid_argument("plan: no pivot in column " + std::to_string(j));
        for (int32_t q = p.col_ptr[j]; q < p.col_ptr[j + 1]; ++q) {
            const int32_t r = p.row_idx[q];
            if (r < 0 || r >= n || (q < p.diag_pos[j] && r >= j) || (q > p.diag_pos[j] && r <= j))
                throw std::invalid_argument("plan: U/L rows out of place in column " +
                                            std::to_string(j));
        }
    }

    // Update map for the left-looking refactor: for U(r, j), the positions
    // in column j of the rows of L(:, r).  Counted first (upd_start), then
    // filled column by column — on several host threads for large plans.
    p.upd_start.assign(p.nnz_lu, 0);
    int64_t total = 0;
    for (int32_t j = 0; j < n; ++j)
        for (int32_t q = p.col_ptr[j]; q < p.diag_pos[j]; ++q) {
            const int32_t r = p.row_idx[q];
            total += p.col_ptr[r + 1] - p.diag_pos[r] - 1;
        }
    p.has_update_map = total <= update_map_limit();
    if (p.has_update_map) {
        int64_t start = 0;
        for (int32_t j = 0; j < n; ++j)
            for (int32_t q = p.col_ptr[j]; q < p.diag_pos[j]; ++q) {
                p.upd_start[q] = static_cast<int32_t>(start);
                const int32_t r = p.row_idx[q];
                start += p.col_ptr[r + 1] - p.diag_pos[r] - 1;
            }
    }
    p.upd_dst.clear();
    if (p.has_update_map) p.upd_dst.resize(static_cast<size_t>(total));  // every entry written below
    // First failing column of each kind (duplicate row / fill not closed),
    // so that the error does not depend on the thread schedule.
    std::atomic<int32_t> bad_dup{INT32_MAX}, bad_fill{INT32_MAX};
    auto fill_columns = [&](std::atomic<int32_t>& next_col, int32_t chunk) {
        std::vector<int32_t> where(n, -1);
        for (;;) {
            const int32_t j0 = next_col.fetch_add(chunk);
            if (j0 >= n) break;
            const int32_t j1 = std::min(n, j0 + chunk);
            for (int32_t j = j0; j < j1; ++j) {
                bool dup = false;
                for (int32_t q = p.col_ptr[j]; q < p.col_ptr[j + 1]; ++q) {
                    if (where[p.row_idx[q]] >= 0) dup = true;
                    where[p.row_idx[q]] = q;
                }
                bool open = false;
                if (!dup) {
                    for (int32_t q = p.col_ptr[j]; q < p.diag_pos[j] && !open; ++q) {
                        const int32_t r = p.row_idx[q];
                        int32_t* out = p.upd_dst.data() + p.upd_start[q];
                        for (int32_t k = p.diag_pos[r] + 1; k < p.col_ptr[r + 1]; ++k) {
                            const int32_t d = where[p.row_idx[k]];
                            if (d < 0) {
                                open = true;
                                break;
                            }
                            *out++ = d - p.col_ptr[j];  // relative to column j
                        }
                    }
                }
                for (int32_t q = p.col_ptr[j]; q < p.col_ptr[j + 1]; ++q) where[p.row_idx[q]] = -1;
                auto lower = [](std::atomic<int32_t>& a, int32_t v) {
                    int32_t cur = a.load();
                    while (v < cur && !a.compare_exchange_weak(cur, v)) {
                    }
                };
                if (dup) lower(bad_dup, j);
                if (open) lower(bad_fill, j);
            }
        }
    };
    if (p.has_update_map) {
        std::atomic<int32_t> next_col{0};
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const int nthreads = total >= (int64_t{1} << 25) ? static_cast<int>(std::min(hw, 16u)) : 1;
        if (nthreads == 1) {
            fill_columns(next_col, n);
        } else {
            std::vector<std::thread> pool;
            for (int t = 0; t < nthreads; ++t) pool.emplace_back(fill_columns, std::ref(next_col), 64);
            for (auto& th : pool) th.join();
        }
    }
    const int32_t first_bad = std::min(bad_dup.load(), bad_fill.load());
    if (first_bad != INT32_MAX) {
        if (bad_dup.load() == first_bad)
            throw std::invalid_argument("plan: duplicate row in column " + std::to_string(first_bad));
        throw std::invalid_argument("plan: fill pattern not closed at column " +
                                    std::to_string(first_bad));
    }
    p.updates = total;
    p.max_col = 0;
    for (int32_t j = 0; j < n; ++j) p.max_col = std::max(p.max_col, p.col_ptr[j + 1] - p.col_ptr[j]);

    // Row-wise L and U.
    std::vector<int32_t> lcount(n + 1, 0), ucount(n + 1, 0);
    for (int32_t j = 0; j < n; ++j)
        for (int32_t q = p.col_ptr[j]; q < p.col_ptr[j + 1]; ++q) {
            const int32_t i = p.row_idx[q];
            if (i > j) ++lcount[i + 1];
            else if (i < j) ++ucount[i + 1];
        }
    for (int32_t i = 0; i < n; ++i) {
        lcount[i + 1] += lcount[i];
        ucount[i + 1] += ucount[i];
    }
    p.lrow_ptr = lcount;
    p.urow_ptr = ucount;
    p.lrow_pos.assign(lcount[n], 0);
    p.lrow_col.assign(lcount[n], 0);
    p.urow_pos.assign(ucount[n], 0);
    p.urow_col.assign(ucount[n], 0);
    std::vector<int32_t> lf(lcount.begin(), lcount.end() - 1), uf(ucount.begin(), ucount.end() - 1);
    for (int32_t j = 0; j < n; ++j)  // columns ascending -> rows get ascending columns
        for (int32_t q = p.col_ptr[j]; q < p.col_ptr[j + 1]; ++q) {
            const int32_t i = p.row_idx[q];
            if (i > j) {
                p.lrow_pos[lf[i]] = q;
                p.lrow_col[lf[i]++] = j;
            } else if (i < j) {
                p.urow_pos[uf[i]] = q;
                p.urow_col[uf[i]++] = j;
            }
        }

    p.umeta.assign(4 * static_cast<size_t>(p.nnz_lu), 0);
    for (int32_t j = 0; j < n; ++j)
        for (int32_t q = p.col_ptr[j]; q < p.diag_pos[j]; ++q) {
            const int32_t r = p.row_idx[q];
            p.umeta[4 * q] = r;
            p.umeta[4 * q + 1] = p.diag_pos[r];
            p.umeta[4 * q + 2] = p.col_ptr[r + 1] - p.diag_pos[r] - 1;
            p.umeta[4 * q + 3] = p.upd_start[q];
        }
    p.rowcopy_pos.assign(p.nnz_lu, -1);
    for (int32_t i = 0; i < n; ++i) {
        for (int32_t k = p.lrow_ptr[i]; k < p.lrow_ptr[i + 1]; ++k) p.rowcopy_pos[p.lrow_pos[k]] = k;
        for (int32_t k = p.urow_ptr[i]; k < p.urow_ptr[i + 1]; ++k) p.rowcopy_pos[p.urow_pos[k]] = k;
    }

    // Level schedules.
    std::vector<int32_t> lev(n, 0);
    for (int32_t j = 0; j < n; ++j) {
        int32_t l = 0;
        for (int32_t q = p.col_ptr[j]; q < p.diag_pos[j]; ++q)
            l = std::max(l, lev[p.row_idx[q]] + 1);
        lev[j] = l;
    }
    level_sort(lev, p.col_lev_ptr, p.col_lev);
    for (int32_t i = 0; i < n; ++i) {
        int32_t l = 0;
        for (int32_t k = p.lrow_ptr[i]; k < p.lrow_ptr[i + 1]; ++k)
            l = std::max(l, lev[p.lrow_col[k]] + 1);
        lev[i] = l;
    }
    level_sort(lev, p.fwd_lev_ptr, p.fwd_lev);
    for (int32_t i = n - 1; i >= 0; --i) {
        int32_t l = 0;
        for (int32_t k = p.urow_ptr[i]; k < p.urow_ptr[i + 1]; ++k)
            l = std::max(l, lev[p.urow_col[k]] + 1);
        lev[i] = l;
    }
    level_sort(lev, p.bwd_lev_ptr, p.bwd_lev);
    for (int32_t i = n - 1; i >= 0; --i) {
        int32_t l = 0;
        for (int32_t q = p.diag_pos[i] + 1; q < p.col_ptr[i + 1]; ++q)
            l = std::max(l, lev[p.row_idx[q]] + 1);
        lev[i] = l;
    }
    level_sort(lev, p.tbw_lev_ptr, p.tbw_lev);

    p.a_to_lu.assign(p.nnz_a, -1);
    for (int32_t q = 0; q < p.nnz_lu; ++q)
        if (p.lu_src[q] >= 0) p.a_to_lu[p.lu_src[q]] = q;
    for (int32_t k = 0; k < p.nnz_a; ++k)
        if (p.a_to_lu[k] < 0)
            throw std::invalid_argument("plan: caller slot without an element");
}

}  // namespace

// Order of the arrays in the device pool; must match PlanArrays in the
// kernels' header.
#define NSG_PLAN_ARRAYS(X)                                                      \
    X(perm_row) X(perm_col) X(col_ptr) X(row_idx) X(diag_pos) X(lu_src)         \
    X(upd_start) X(upd_dst) X(lrow_ptr) X(lrow_pos) X(lrow_col) X(urow_ptr)     \
    X(urow_pos) X(urow_col) X(col_lev_ptr) X(col_lev) X(fwd_lev_ptr) X(fwd_lev) \
    X(bwd_lev_ptr) X(bwd_lev) X(tbw_lev_ptr) X(tbw_lev) X(rowcopy_pos) X(umeta) \
    X(piv_rank) X(gmin_pos)

namespace {
template <class V>
bool is_update_map(const TopologyPlan& p, const V& v) {
    return static_cast<const void*>(&v) == static_cast<const void*>(&p.upd_dst);
}

// v's values (each below 65,536) as consecutive uint16, in ceil(|v| / 2)
// words; the last half word of an odd count is zero.
template <class V>
void append_packed16(std::vector<int32_t>& pool, const V& v) {
    const size_t at = pool.size();
    pool.resize(at + (v.size() + 1) / 2, 0);
    char* out = reinterpret_cast<char*>(pool.data() + at);
    uint16_t chunk[4096];
    for (size_t k0 = 0; k0 < v.size(); k0 += 4096) {
        const size_t m = std::min<size_t>(4096, v.size() - k0);
        for (size_t k = 0; k < m; ++k) chunk[k] = static_cast<uint16_t>(v[k0 + k]);
        std::memcpy(out + 2 * k0, chunk, 2 * m);
    }
}
}  // namespace

// A packed update map takes one int32 word per two positions.
int64_t TopologyPlan::device_words() const {
    int64_t w = 0;
#define NSG_COUNT(name)                                                          \
    w += (is_update_map(*this, name) && map16() ? (static_cast<int64_t>(name.size()) + 1) / 2 \
                                                 : static_cast<int64_t>(name.size())) +       \
         4;  // 16 B align
    NSG_PLAN_ARRAYS(NSG_COUNT)
#undef NSG_COUNT
    return w;
}

void TopologyPlan::append_to(std::vector<int32_t>& pool, int64_t* off) const {
    int idx = 0;
    const bool pack = map16();
#define NSG_APPEND(name)                                          \
    while (pool.size() % 4) pool.push_back(0);                    \
    off[idx++] = static_cast<int64_t>(pool.size());               \
    if (pack && is_update_map(*this, name)) {                     \
        append_packed16(pool, name);                              \
    } else {                                                      \
        pool.insert(pool.end(), name.begin(), name.end());        \
    }
    NSG_PLAN_ARRAYS(NSG_APPEND)
#undef NSG_APPEND
}

TopologyPlan build_plan(const MarkowitzOrder& mo, const std::vector<int32_t>& slot_elem) {
    TopologyPlan p;
    p.n = mo.size();
    p.nnz_a = static_cast<int32_t>(slot_elem.size());
    p.perm_row.resize(p.n);
    p.perm_col.resize(p.n);
    for (int32_t i = 1; i <= p.n; ++i) {
        p.perm_row[i - 1] = mo.int_to_ext_row()[i] - 1;
        p.perm_col[i - 1] = mo.int_to_ext_col()[i] - 1;
    }
    std::vector<int32_t> slot_of(mo.element_count(), -1);
    for (int32_t k = 0; k < p.nnz_a; ++k) slot_of[slot_elem[k]] = k;
    p.col_ptr.assign(p.n + 1, 0);
    for (int32_t j = 1; j <= p.n; ++j) {
        for (int32_t e = mo.first_in_col(j); e >= 0; e = mo.next_in_col(e)) {
            p.row_idx.push_back(mo.row_of(e) - 1);
            p.lu_src.push_back(slot_of[e]);
        }
        p.col_ptr[j] = static_cast<int32_t>(p.row_idx.size());
    }
    finish(p);
    return p;
}

TopologyPlan build_plan_amd(const AmdLuFactor& f) {
    if (!f.factored()) throw std::logic_error("build_plan_amd: engine not factored");
    TopologyPlan p;
    p.kind = kPlanKindAmdLu;
    p.n = f.size();
    p.nnz_a = f.nnz();
    const int32_t n = p.n;
    const auto& q = f.q();
    const auto& pinv = f.pinv();
    const auto& acp = f.col_ptr();
    const auto& ari = f.row_idx();
    p.perm_row.assign(n, -1);
    for (int32_t r = 0; r < n; ++r) p.perm_row[pinv[r]] = r;
    p.perm_col = q;
    p.piv_rank = f.piv_rank();
    p.gmin_pos.assign(n, -1);
    p.col_ptr.assign(n + 1, 0);
    p.row_idx.reserve(f.Li().size() + f.Ui().size());
    p.lu_src.reserve(f.Li().size() + f.Ui().size());
    std::vector<int32_t> slot_at(n, -1);  // pivot-step row -> A slot of this column
    for (int32_t k = 0; k < n; ++k) {
        const int32_t col = q[k];
        for (int32_t a = acp[col]; a < acp[col + 1]; ++a) slot_at[pinv[ari[a]]] = a;
        const int32_t c0 = static_cast<int32_t>(p.row_idx.size());
        auto push = [&](int32_t s) {
            if (s == pinv[col]) p.gmin_pos[k] = static_cast<int32_t>(p.row_idx.size()) - c0;
            p.row_idx.push_back(s);
            p.lu_src.push_back(slot_at[s]);
        };
        // U(:, k) above the pivot in replay order, the pivot (stored last in
        // U(:, k) by the reference), then L(:, k) after its unit diagonal.
        for (int32_t u = f.Up()[k]; u < f.Up()[k + 1] - 1; ++u) push(f.Ui()[u]);
        push(k);
        for (int32_t l = f.Lp()[k] + 1; l < f.Lp()[k + 1]; ++l) push(f.Li()[l]);
        for (int32_t a = acp[col]; a < acp[col + 1]; ++a) slot_at[pinv[ari[a]]] = -1;
        p.col_ptr[k + 1] = static_cast<int32_t>(p.row_idx.size());
    }
    finish(p);
    return p;
}

TopologyPlan build_plan_from_structure(int32_t n, int32_t nnz_a,
                                       const int32_t* int_to_ext_row,
                                       const int32_t* int_to_ext_col,
                                       int32_t n_elem, const int32_t* elem_row,
                                       const int32_t* elem_col,
                                       const int32_t* slot_to_elem) {
    if (n <= 0 || nnz_a <= 0 || n_elem < nnz_a)
        throw std::invalid_argument("plan: bad sizes");
    TopologyPlan p;
    p.n = n;
    p.nnz_a = nnz_a;
    p.perm_row.resize(n);
    p.perm_col.resize(n);
    for (int32_t i = 0; i < n; ++i) {
        if (int_to_ext_row[i] < 1 || int_to_ext_row[i] > n || int_to_ext_col[i] < 1 ||
            int_to_ext_col[i] > n)
            throw std::invalid_argument("plan: permutation out of range");
        p.perm_row[i] = int_to_ext_row[i] - 1;
        p.perm_col[i] = int_to_ext_col[i] - 1;
    }
    std::vector<int32_t> slot_of(n_elem, -1);
    for (int32_t k = 0; k < nnz_a; ++k) {
        if (slot_to_elem[k] < 0 || slot_to_elem[k] >= n_elem)
            throw std::invalid_argument("plan: slot map out of range");
        slot_of[slot_to_elem[k]] = k;
    }
    p.col_ptr.assign(n + 1, 0);
    p.row_idx.resize(n_elem);
    p.lu_src.resize(n_elem);
    for (int32_t e = 0; e < n_elem; ++e) {
        if (elem_col[e] < 1 || elem_col[e] > n || elem_row[e] < 1 || elem_row[e] > n ||
            (e > 0 && elem_col[e] < elem_col[e - 1]))
            throw std::invalid_argument("plan: element list not column ordered");
        ++p.col_ptr[elem_col[e]];
        p.row_idx[e] = elem_row[e] - 1;
        p.lu_src[e] = slot_of[e];
    }
    for (int32_t j = 0; j < n; ++j) p.col_ptr[j + 1] += p.col_ptr[j];
    finish(p);
    return p;
}

}  // namespace nsg
