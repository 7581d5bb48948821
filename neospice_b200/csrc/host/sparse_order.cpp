// Sparse-1.3-compatible Markowitz ordering (host symbolic phase).
// Each routine names the reference routine whose pivot-selection behaviour it
// must reproduce; the storage (index pool, sorted singly linked lists) and the
// list maintenance are this project's own.
#include "sparse_order.hpp"

#include <algorithm>
#include <climits>
#include <cmath>
#include <stdexcept>

namespace nsg {

namespace {
constexpr int32_t kNone = -1;
constexpr int32_t kLargestShort = 32767;   // SHRT_MAX, src/solver/config.hpp:37
constexpr long kLargestLong = LONG_MAX;    // src/solver/config.hpp:38
constexpr long kTiesMultiplier = 5;        // src/solver/config.hpp:26
constexpr int32_t kMinAllocated = 6;       // src/solver/config.hpp:22
}  // namespace

MarkowitzOrder::MarkowitzOrder(int32_t size) : size_(size) {
    if (size < 0) throw std::invalid_argument("MarkowitzOrder: negative size");
    const int32_t alloc = std::max(size, kMinAllocated);
    first_in_col_.assign(alloc + 1, kNone);
    first_in_row_.assign(alloc + 1, kNone);
    diag_.assign(alloc + 1, kNone);
    int_to_ext_row_.resize(alloc + 1);
    int_to_ext_col_.resize(alloc + 1);
    for (int32_t i = 0; i <= alloc; ++i) int_to_ext_row_[i] = int_to_ext_col_[i] = i;
    ext_to_int_row_.assign(alloc + 1, -1);
    ext_to_int_col_.assign(alloc + 1, -1);
    ext_to_int_row_[0] = ext_to_int_col_[0] = 0;
    pool_.reserve(static_cast<size_t>(alloc) * 10);
}

// element_mag: |re| + |im| (the imaginary part stays 0 for real values).
double MarkowitzOrder::mag(int32_t e) const {
    return std::fabs(pool_[e].val) + std::fabs(pool_[e].imag);
}

// External indices get internal numbers in order of first appearance, row
// index before column index (src/solver/build.cpp:197-249).
void MarkowitzOrder::translate(int32_t& row, int32_t& col) {
    auto intern = [&](int32_t ext) {
        if (ext >= static_cast<int32_t>(ext_to_int_row_.size()))
            throw std::out_of_range("MarkowitzOrder: external index beyond size");
        if (ext_to_int_row_[ext] == -1) {
            const int32_t k = ++current_size_;
            if (k > size_) throw std::out_of_range("MarkowitzOrder: too many indices");
            ext_to_int_row_[ext] = ext_to_int_col_[ext] = k;
            int_to_ext_row_[k] = int_to_ext_col_[k] = ext;
        }
    };
    intern(row);
    const int32_t r = ext_to_int_row_[row];
    intern(col);
    row = r;
    col = ext_to_int_col_[col];
}

int32_t MarkowitzOrder::new_element(int32_t row, int32_t col, bool fill) {
    Element el;
    el.row = row;
    el.col = col;
    el.fill = fill;
    pool_.push_back(el);
    const int32_t e = static_cast<int32_t>(pool_.size()) - 1;
    if (row == col) diag_[row] = e;
    return e;
}

// Keep column lists sorted by row.
void MarkowitzOrder::insert_in_col(int32_t e, int32_t col) {
    const int32_t row = pool_[e].row;
    int32_t prev = kNone, cur = first_in_col_[col];
    while (cur != kNone && pool_[cur].row < row) {
        prev = cur;
        cur = pool_[cur].next_in_col;
    }
    pool_[e].next_in_col = cur;
    if (prev == kNone) first_in_col_[col] = e;
    else pool_[prev].next_in_col = e;
}

// Keep row lists sorted by column.
void MarkowitzOrder::insert_in_row(int32_t e, int32_t row) {
    const int32_t col = pool_[e].col;
    int32_t prev = kNone, cur = first_in_row_[row];
    while (cur != kNone && pool_[cur].col < col) {
        prev = cur;
        cur = pool_[cur].next_in_row;
    }
    pool_[e].next_in_row = cur;
    if (prev == kNone) first_in_row_[row] = e;
    else pool_[prev].next_in_row = e;
}

int32_t MarkowitzOrder::find_in_col(int32_t col, int32_t row) const {
    for (int32_t e = first_in_col_[col]; e != kNone; e = pool_[e].next_in_col) {
        if (pool_[e].row == row) return e;
        if (pool_[e].row > row) break;
    }
    return kNone;
}

int32_t MarkowitzOrder::get_element(int32_t ext_row, int32_t ext_col) {
    if (rows_linked_) throw std::logic_error("MarkowitzOrder: pattern is frozen");
    if (ext_row <= 0 || ext_col <= 0)
        throw std::invalid_argument("MarkowitzOrder: ground has no element");
    int32_t row = ext_row, col = ext_col;
    translate(row, col);
    if (row == col && diag_[row] != kNone) return diag_[row];
    int32_t e = find_in_col(col, row);
    if (e != kNone) return e;
    e = new_element(row, col, false);
    insert_in_col(e, col);
    needs_ordering_ = true;
    return e;
}

void MarkowitzOrder::clear_fillins() {
    for (auto& el : pool_)
        if (el.fill) el.val = el.imag = 0.0;
}

// --- MNA pre-ordering: swap +-1 "twin" columns so that a voltage source's
// branch row gets a structural diagonal (src/solver/utils.cpp:8-89).

int32_t MarkowitzOrder::count_twins(int32_t col, int32_t& t1, int32_t& t2) {
    int32_t twins = 0;
    for (int32_t a = first_in_col_[col]; a != kNone; a = pool_[a].next_in_col) {
        if (std::fabs(pool_[a].val) != 1.0) continue;
        const int32_t row = pool_[a].row;
        int32_t b = first_in_col_[row];
        while (b != kNone && pool_[b].row != col) b = pool_[b].next_in_col;
        if (b != kNone && std::fabs(pool_[b].val) == 1.0) {
            if (++twins >= 2) return twins;
            t1 = a;
            pool_[a].col = col;
            t2 = b;
            pool_[b].col = row;
        }
    }
    return twins;
}

void MarkowitzOrder::swap_cols(int32_t t1, int32_t t2) {
    const int32_t c1 = pool_[t1].col, c2 = pool_[t2].col;
    std::swap(first_in_col_[c1], first_in_col_[c2]);
    std::swap(int_to_ext_col_[c1], int_to_ext_col_[c2]);
    ext_to_int_col_[int_to_ext_col_[c2]] = c2;
    ext_to_int_col_[int_to_ext_col_[c1]] = c1;
    diag_[c1] = t2;
    diag_[c2] = t1;
}

void MarkowitzOrder::mna_preorder() {
    if (rows_linked_ || preordered_) return;
    preordered_ = true;
    int32_t start_at = 1;
    bool another_pass;
    do {
        another_pass = false;
        bool swapped = false;
        for (int32_t j = start_at; j <= size_; ++j) {
            if (diag_[j] != kNone) continue;
            int32_t t1 = kNone, t2 = kNone;
            const int32_t twins = count_twins(j, t1, t2);
            if (twins == 1) {
                swap_cols(t1, t2);
                swapped = true;
            } else if (twins > 1 && !another_pass) {
                another_pass = true;
                start_at = j;
            }
        }
        if (another_pass) {
            // Break a multi-twin deadlock with the first twin pair of the
            // first column still lacking a diagonal.
            for (int32_t j = start_at; !swapped && j <= size_; ++j) {
                if (diag_[j] != kNone) continue;
                int32_t t1 = kNone, t2 = kNone;
                if (count_twins(j, t1, t2) >= 1 && t1 != kNone) {
                    swap_cols(t1, t2);
                    swapped = true;
                }
            }
            if (!swapped) break;
        }
    } while (another_pass);
}

void MarkowitzOrder::add_diag_gmin(double gmin) {
    if (gmin == 0.0) return;
    for (int32_t i = size_; i > 0; --i)
        if (diag_[i] != kNone) pool_[diag_[i]].val += gmin;
}

// Build row lists from the column lists; columns are visited last to first
// and prepended so each row list ends sorted by column
// (src/solver/build.cpp:183-195).
void MarkowitzOrder::link_rows() {
    std::fill(first_in_row_.begin(), first_in_row_.end(), kNone);
    for (int32_t col = size_; col >= 1; --col) {
        for (int32_t e = first_in_col_[col]; e != kNone; e = pool_[e].next_in_col) {
            pool_[e].col = col;
            pool_[e].next_in_row = first_in_row_[pool_[e].row];
            first_in_row_[pool_[e].row] = e;
        }
    }
    rows_linked_ = true;
}

// --- Markowitz bookkeeping (src/solver/factor.cpp:61-115) ---

void MarkowitzOrder::count_markowitz(int32_t step) {
    for (int32_t i = step; i <= size_; ++i) {
        int32_t count = -1;
        for (int32_t e = first_in_row_[i]; e != kNone; e = pool_[e].next_in_row)
            if (pool_[e].col >= step) ++count;
        mrow_[i] = count;
    }
    for (int32_t i = step; i <= size_; ++i) {
        int32_t count = -1;
        for (int32_t e = first_in_col_[i]; e != kNone; e = pool_[e].next_in_col)
            if (pool_[e].row >= step) ++count;
        mcol_[i] = count;
    }
}

long MarkowitzOrder::product_of(int32_t r, int32_t c) const {
    if ((r > kLargestShort && c != 0) || (c > kLargestShort && r != 0)) {
        const double fp = static_cast<double>(r) * static_cast<double>(c);
        return fp >= static_cast<double>(kLargestLong) ? kLargestLong : static_cast<long>(fp);
    }
    return static_cast<long>(r) * c;
}

void MarkowitzOrder::markowitz_products(int32_t step) {
    singletons_ = 0;
    for (int32_t i = step; i <= size_; ++i) {
        const int32_t r = mrow_[i], c = mcol_[i];
        if ((r > kLargestShort && c != 0) || (c > kLargestShort && r != 0)) {
            mprod_[i] = product_of(r, c);
        } else {
            mprod_[i] = static_cast<long>(r) * c;
            if (mprod_[i] == 0) ++singletons_;
        }
    }
}

// --- Column magnitude scans (src/solver/factor.cpp:28-55) ---

double MarkowitzOrder::largest_in_col_from(int32_t e) const {
    double largest = 0.0;
    for (; e != kNone; e = pool_[e].next_in_col)
        if (mag(e) > largest) largest = mag(e);
    return largest;
}

double MarkowitzOrder::largest_in_col_excluding(int32_t pe, int32_t step) const {
    const int32_t row = pool_[pe].row;
    int32_t e = first_in_col_[pool_[pe].col];
    while (e != kNone && pool_[e].row < step) e = pool_[e].next_in_col;
    double largest = (pool_[e].row != row) ? mag(e) : 0.0;
    for (e = pool_[e].next_in_col; e != kNone; e = pool_[e].next_in_col)
        if (mag(e) > largest && pool_[e].row != row) largest = mag(e);
    return largest;
}

// --- Pivot search, in the reference's order: singletons, quick diagonal,
// full diagonal, whole matrix (src/solver/factor.cpp:121-396) ---

int32_t MarkowitzOrder::search_singleton(int32_t step) {
    mprod_[size_ + 1] = mprod_[step];
    mprod_[step - 1] = 0;
    int32_t remaining = singletons_--;
    int32_t scan = size_ + 1;
    while (remaining-- > 0) {
        while (mprod_[scan] != 0) --scan;
        int32_t i = scan--;
        if (i < step) break;
        if (i > size_) i = step;
        const int32_t d = diag_[i];
        if (d != kNone) {
            const double pm = mag(d);
            if (pm > abs_threshold_ &&
                pm > rel_threshold_ * largest_in_col_excluding(d, step))
                return d;
            continue;
        }
        // The candidate's only reduced entry is off the diagonal: the
        // reference abandons the singleton search here.
        break;
    }
    ++singletons_;
    return kNone;
}

int32_t MarkowitzOrder::search_diagonal_quick(int32_t step) {
    int32_t chosen = kNone;
    long min_product = kLargestLong;
    mprod_[size_ + 1] = mprod_[step];
    mprod_[step - 1] = -1;
    int32_t scan = size_ + 2;
    for (;;) {
        --scan;
        while (mprod_[scan] >= min_product) --scan;
        int32_t i = scan;
        if (i < step) break;
        if (i > size_) i = step;
        const int32_t d = diag_[i];
        if (d == kNone) continue;
        const double m = mag(d);
        if (m <= abs_threshold_) continue;
        if (mprod_[scan] == 1) {
            // Product 1: a 2x2 symmetric block; accept at once when the
            // diagonal dominates its two partners.
            int32_t in_row = pool_[d].next_in_row;
            int32_t in_col = pool_[d].next_in_col;
            if (in_row == kNone && in_col == kNone) {
                in_row = first_in_row_[i];
                while (in_row != kNone &&
                       !(pool_[in_row].col >= step && pool_[in_row].col != i))
                    in_row = pool_[in_row].next_in_row;
                in_col = first_in_col_[i];
                while (in_col != kNone &&
                       !(pool_[in_col].row >= step && pool_[in_col].row != i))
                    in_col = pool_[in_col].next_in_col;
            }
            if (in_row != kNone && in_col != kNone &&
                pool_[in_row].col == pool_[in_col].row) {
                const double off = std::max(mag(in_row), mag(in_col));
                if (m >= off) return d;
            }
        }
        min_product = mprod_[scan];
        chosen = d;
    }
    if (chosen != kNone &&
        mag(chosen) <= rel_threshold_ * largest_in_col_excluding(chosen, step))
        chosen = kNone;
    return chosen;
}

int32_t MarkowitzOrder::search_diagonal_full(int32_t step) {
    int32_t chosen = kNone;
    long min_product = kLargestLong;
    long ties = 0;
    double accepted_ratio = 0.0;
    mprod_[size_ + 1] = mprod_[step];
    for (int32_t j = size_ + 1; j > step; --j) {
        if (mprod_[j] > min_product) continue;
        const int32_t i = (j > size_) ? step : j;
        const int32_t d = diag_[i];
        if (d == kNone) continue;
        const double m = mag(d);
        if (m <= abs_threshold_) continue;
        const double largest = largest_in_col_excluding(d, step);
        if (m <= rel_threshold_ * largest) continue;
        if (mprod_[j] < min_product) {
            chosen = d;
            min_product = mprod_[j];
            accepted_ratio = largest / m;
            ties = 0;
        } else {
            ++ties;
            const double ratio = largest / m;
            if (ratio < accepted_ratio) {
                chosen = d;
                accepted_ratio = ratio;
            }
            if (ties >= min_product * kTiesMultiplier) return chosen;
        }
    }
    return chosen;
}

int32_t MarkowitzOrder::search_whole(int32_t step) {
    int32_t chosen = kNone, biggest = kNone;
    double biggest_mag = 0.0;
    long min_product = kLargestLong;
    long ties = 0;
    double accepted_ratio = 0.0;
    for (int32_t i = step; i <= size_; ++i) {
        int32_t e = first_in_col_[i];
        while (e != kNone && pool_[e].row < step) e = pool_[e].next_in_col;
        const double largest = largest_in_col_from(e);
        if (largest == 0.0) continue;
        for (; e != kNone; e = pool_[e].next_in_col) {
            const double m = mag(e);
            if (m > biggest_mag) {
                biggest_mag = m;
                biggest = e;
            }
            const long product =
                static_cast<long>(mrow_[pool_[e].row]) * mcol_[pool_[e].col];
            if (product <= min_product && m > rel_threshold_ * largest &&
                m > abs_threshold_) {
                if (product < min_product) {
                    chosen = e;
                    min_product = product;
                    accepted_ratio = largest / m;
                    ties = 0;
                } else {
                    ++ties;
                    const double ratio = largest / m;
                    if (ratio < accepted_ratio) {
                        chosen = e;
                        accepted_ratio = ratio;
                    }
                    if (ties >= min_product * kTiesMultiplier) return chosen;
                }
            }
        }
    }
    if (chosen != kNone) return chosen;
    if (biggest_mag == 0.0) {
        error_ = OrderStatus::singular;
        return kNone;
    }
    return biggest;  // SmallPivot, which the reference reports as OK
}

int32_t MarkowitzOrder::search_for_pivot(int32_t step, bool diag_pivoting) {
    if (singletons_) {
        const int32_t p = search_singleton(step);
        if (p != kNone) return p;
    }
    if (diag_pivoting) {
        int32_t p = search_diagonal_quick(step);
        if (p != kNone) return p;
        p = search_diagonal_full(step);
        if (p != kNone) return p;
    }
    return search_whole(step);
}

// --- Row and column interchange.  Lists stay sorted, so relabelling two
// rows (columns) and re-sorting the touched column (row) lists reproduces the
// reference's list order after row_exchange / col_exchange
// (src/solver/factor.cpp:402-640). ---

void MarkowitzOrder::swap_rows(int32_t r1, int32_t r2) {
    if (r1 > r2) std::swap(r1, r2);
    // Columns touched: union of the two row lists.
    int32_t a = first_in_row_[r1], b = first_in_row_[r2];
    while (a != kNone || b != kNone) {
        int32_t col;
        int32_t e1 = kNone, e2 = kNone;
        if (b == kNone || (a != kNone && pool_[a].col < pool_[b].col)) {
            col = pool_[a].col;
            e1 = a;
            a = pool_[a].next_in_row;
        } else if (a == kNone || pool_[a].col > pool_[b].col) {
            col = pool_[b].col;
            e2 = b;
            b = pool_[b].next_in_row;
        } else {
            col = pool_[a].col;
            e1 = a;
            e2 = b;
            a = pool_[a].next_in_row;
            b = pool_[b].next_in_row;
        }
        // Unlink e1/e2 from column col, relabel, re-insert in order.
        int32_t prev = kNone, cur = first_in_col_[col];
        while (cur != kNone) {
            const int32_t nxt = pool_[cur].next_in_col;
            if (cur == e1 || cur == e2) {
                if (prev == kNone) first_in_col_[col] = nxt;
                else pool_[prev].next_in_col = nxt;
            } else {
                prev = cur;
            }
            if (pool_[cur].row >= r2) break;
            cur = nxt;
        }
        if (e1 != kNone) {
            pool_[e1].row = r2;
        }
        if (e2 != kNone) {
            pool_[e2].row = r1;
            insert_in_col(e2, col);
        }
        if (e1 != kNone) insert_in_col(e1, col);
    }
    std::swap(mrow_[r1], mrow_[r2]);
    std::swap(first_in_row_[r1], first_in_row_[r2]);
    std::swap(int_to_ext_row_[r1], int_to_ext_row_[r2]);
    ext_to_int_row_[int_to_ext_row_[r1]] = r1;
    ext_to_int_row_[int_to_ext_row_[r2]] = r2;
}

void MarkowitzOrder::swap_columns(int32_t c1, int32_t c2) {
    if (c1 > c2) std::swap(c1, c2);
    int32_t a = first_in_col_[c1], b = first_in_col_[c2];
    while (a != kNone || b != kNone) {
        int32_t row;
        int32_t e1 = kNone, e2 = kNone;
        if (b == kNone || (a != kNone && pool_[a].row < pool_[b].row)) {
            row = pool_[a].row;
            e1 = a;
            a = pool_[a].next_in_col;
        } else if (a == kNone || pool_[a].row > pool_[b].row) {
            row = pool_[b].row;
            e2 = b;
            b = pool_[b].next_in_col;
        } else {
            row = pool_[a].row;
            e1 = a;
            e2 = b;
            a = pool_[a].next_in_col;
            b = pool_[b].next_in_col;
        }
        int32_t prev = kNone, cur = first_in_row_[row];
        while (cur != kNone) {
            const int32_t nxt = pool_[cur].next_in_row;
            if (cur == e1 || cur == e2) {
                if (prev == kNone) first_in_row_[row] = nxt;
                else pool_[prev].next_in_row = nxt;
            } else {
                prev = cur;
            }
            if (pool_[cur].col >= c2) break;
            cur = nxt;
        }
        if (e1 != kNone) pool_[e1].col = c2;
        if (e2 != kNone) {
            pool_[e2].col = c1;
            insert_in_row(e2, row);
        }
        if (e1 != kNone) insert_in_row(e1, row);
    }
    std::swap(mcol_[c1], mcol_[c2]);
    std::swap(first_in_col_[c1], first_in_col_[c2]);
    std::swap(int_to_ext_col_[c1], int_to_ext_col_[c2]);
    ext_to_int_col_[int_to_ext_col_[c1]] = c1;
    ext_to_int_col_[int_to_ext_col_[c2]] = c2;
}

// Move the pivot to (step, step) and keep Markowitz products and the
// singleton count consistent (src/solver/factor.cpp:642-700).
void MarkowitzOrder::exchange(int32_t pivot, int32_t step) {
    const int32_t row = pool_[pivot].row, col = pool_[pivot].col;
    if (row == step && col == step) return;
    auto singleton_delta = [&](long now, long before) {
        if ((now == 0) != (before == 0)) {
            if (before == 0) --singletons_;
            else ++singletons_;
        }
    };
    if (row == col) {
        swap_rows(step, row);
        swap_columns(step, col);
        std::swap(mprod_[step], mprod_[row]);
        std::swap(diag_[row], diag_[step]);
        return;
    }
    const long before_step = mprod_[step];
    const long before_row = mprod_[row];
    const long before_col = mprod_[col];
    if (row != step) {
        swap_rows(step, row);
        mprod_[row] = static_cast<long>(mrow_[row]) * mcol_[row];
        singleton_delta(mprod_[row], before_row);
    }
    if (col != step) {
        swap_columns(step, col);
        mprod_[col] = static_cast<long>(mcol_[col]) * mrow_[col];
        singleton_delta(mprod_[col], before_col);
        diag_[col] = find_in_col(col, col);
    }
    if (row != step) diag_[row] = find_in_col(row, row);
    diag_[step] = find_in_col(step, step);
    mprod_[step] = static_cast<long>(mcol_[step]) * mrow_[step];
    singleton_delta(mprod_[step], before_step);
}

int32_t MarkowitzOrder::create_fillin(int32_t row, int32_t col) {
    const int32_t e = new_element(row, col, true);
    ++fillins_;
    insert_in_col(e, col);
    insert_in_row(e, row);
    mprod_[row] = static_cast<long>(++mrow_[row]) * mcol_[row];
    if (mrow_[row] == 1 && mcol_[row] != 0) --singletons_;
    mprod_[col] = static_cast<long>(++mcol_[col]) * mrow_[col];
    if (mrow_[col] != 0 && mcol_[col] == 1) --singletons_;
    return e;
}

// Right-looking elimination of one pivot, creating fill-ins
// (src/solver/factor.cpp:735-767).  U(r, c) = a(r, c) * (1 / pivot);
// a(i, c) -= U(r, c) * L(i, r) for every L entry below the pivot.
void MarkowitzOrder::eliminate(int32_t pivot) {
    if (std::fabs(pool_[pivot].val) == 0.0) {
        error_ = OrderStatus::singular;
        return;
    }
    pool_[pivot].val = 1.0 / pool_[pivot].val;
    const double rp = pool_[pivot].val;
    for (int32_t up = pool_[pivot].next_in_row; up != kNone; up = pool_[up].next_in_row) {
        pool_[up].val *= rp;
        const double u = pool_[up].val;
        const int32_t ucol = pool_[up].col;
        int32_t sub = pool_[up].next_in_col;
        for (int32_t lo = pool_[pivot].next_in_col; lo != kNone; lo = pool_[lo].next_in_col) {
            const int32_t row = pool_[lo].row;
            while (sub != kNone && pool_[sub].row < row) sub = pool_[sub].next_in_col;
            if (sub == kNone || pool_[sub].row > row) sub = create_fillin(row, ucol);
            pool_[sub].val -= u * pool_[lo].val;
            sub = pool_[sub].next_in_col;
        }
    }
}

// Complex right-looking elimination (src/solver/factor.cpp:769-806): the
// pivot replaced by its reciprocal (complex_ops::reciprocal), U(r, c) *=
// that reciprocal (mult_assign), a(i, c) -= U(r, c) * L(i, r)
// (mult_subt_assign), each with the reference's operand grouping.
void MarkowitzOrder::eliminate_complex(int32_t pivot) {
    Element& pv = pool_[pivot];
    if (std::fabs(pv.val) + std::fabs(pv.imag) == 0.0) {
        error_ = OrderStatus::singular;
        return;
    }
    {
        const double den_r = pv.val, den_i = pv.imag;
        if ((den_r >= den_i && den_r > -den_i) || (den_r < den_i && den_r <= -den_i)) {
            const double r = den_i / den_r;
            pv.val = 1.0 / (den_r + r * den_i);
            pv.imag = -r * pv.val;
        } else {
            const double r = den_r / den_i;
            pv.imag = -1.0 / (den_i + r * den_r);
            pv.val = -r * pv.imag;
        }
    }
    const double pr = pool_[pivot].val, pi = pool_[pivot].imag;
    for (int32_t up = pool_[pivot].next_in_row; up != kNone; up = pool_[up].next_in_row) {
        {
            const double tmp = pool_[up].val;
            pool_[up].val = tmp * pr - pool_[up].imag * pi;
            pool_[up].imag = tmp * pi + pool_[up].imag * pr;
        }
        const double ur = pool_[up].val, ui = pool_[up].imag;
        const int32_t ucol = pool_[up].col;
        int32_t sub = pool_[up].next_in_col;
        for (int32_t lo = pool_[pivot].next_in_col; lo != kNone; lo = pool_[lo].next_in_col) {
            const int32_t row = pool_[lo].row;
            while (sub != kNone && pool_[sub].row < row) sub = pool_[sub].next_in_col;
            if (sub == kNone || pool_[sub].row > row) sub = create_fillin(row, ucol);
            const double lr = pool_[lo].val, li = pool_[lo].imag;
            pool_[sub].val -= ur * lr - ui * li;
            pool_[sub].imag -= ur * li + ui * lr;
            sub = pool_[sub].next_in_col;
        }
    }
}

void MarkowitzOrder::update_markowitz(int32_t pivot) {
    for (int32_t e = pool_[pivot].next_in_col; e != kNone; e = pool_[e].next_in_col) {
        const int32_t row = pool_[e].row;
        --mrow_[row];
        mprod_[row] = product_of(mrow_[row], mcol_[row]);
        if (mrow_[row] == 0) ++singletons_;
    }
    for (int32_t e = pool_[pivot].next_in_row; e != kNone; e = pool_[e].next_in_row) {
        const int32_t col = pool_[e].col;
        --mcol_[col];
        mprod_[col] = product_of(mrow_[col], mcol_[col]);
        if (mcol_[col] == 0 && mrow_[col] != 0) ++singletons_;
    }
}

OrderStatus MarkowitzOrder::order_and_factor(double rel_threshold, double abs_threshold,
                                             bool diag_pivoting) {
    error_ = OrderStatus::ok;
    reorder_step_ = 0;
    if (rel_threshold <= 0.0 || rel_threshold > 1.0) rel_threshold = rel_threshold_;
    rel_threshold_ = rel_threshold;
    if (abs_threshold < 0.0) abs_threshold = abs_threshold_;
    abs_threshold_ = abs_threshold;

    int32_t step = 1;
    if (!needs_ordering_) {
        // Re-validate the previous pivot sequence step by step.
        bool reorder = false;
        for (step = 1; step <= size_; ++step) {
            const int32_t p = diag_[step];
            if (p == kNone) {
                reorder = true;
                break;
            }
            const double largest = largest_in_col_from(pool_[p].next_in_col);
            if (largest * rel_threshold < mag(p)) {
                if (complex_) eliminate_complex(p);
                else eliminate(p);
            } else {
                reorder = true;
                break;
            }
        }
        if (!reorder) {
            needs_ordering_ = false;
            return error_;
        }
        reorder_step_ = step;
    } else {
        if (!rows_linked_) link_rows();
        if (mrow_.empty()) {
            mrow_.assign(size_ + 1, 0);
            mcol_.assign(size_ + 1, 0);
            mprod_.assign(size_ + 2, 0);
        }
    }

    count_markowitz(step);
    markowitz_products(step);
    for (; step <= size_; ++step) {
        const int32_t p = search_for_pivot(step, diag_pivoting);
        if (p == kNone) return error_ = OrderStatus::singular;
        exchange(p, step);
        if (complex_) eliminate_complex(p);
        else eliminate(p);
        if (error_ != OrderStatus::ok) return error_;
        update_markowitz(p);
    }
    needs_ordering_ = false;
    return error_;
}

}  // namespace nsg
