// Host-side symbolic phase: a Sparse-1.3-compatible Markowitz ordering engine.
//
// This is the setup step of the GPU solver.  It must choose, for the same
// pattern and values, exactly the pivots the reference's SparseMatrix chooses
// (src/solver/factor.cpp:911-978), because the GPU refactor replays that pivot
// sequence and its rounding.  The search order, tie-breaking rules and
// thresholds therefore follow Kundert's published Sparse 1.3 algorithm step
// for step; the data structure is this project's own: an index-based element
// pool with orthogonal singly linked row and column lists kept sorted by
// internal index.
//
// Indices follow the reference's convention: external and internal indices are
// 1-based, index 0 is ground.
#pragma once
#include <cstdint>
#include <vector>

namespace nsg {

enum class OrderStatus : int {
    ok = 0,          // SparseError::OK (src/solver/error.hpp:6)
    no_memory = 8,   // SparseError::NoMemory
    singular = 102,  // SparseError::Singular / ZeroDiag
};

class MarkowitzOrder {
public:
    // SparseMatrix(size) as NeoSolver::symbolic builds it
    // (src/solver/matrix.cpp:7-41, neo_solver.cpp:113-146).
    explicit MarkowitzOrder(int32_t size);

    // SparseMatrix::get_element (src/solver/build.cpp:55-80) for 1-based
    // external (row, col); returns the element id.  Only valid before the
    // first ordering.
    int32_t get_element(int32_t ext_row, int32_t ext_col);

    // Values of element ids (real part, and imaginary part in complex mode).
    double& value(int32_t e) { return pool_[e].val; }
    double value(int32_t e) const { return pool_[e].val; }
    double& value_imag(int32_t e) { return pool_[e].imag; }
    double value_imag(int32_t e) const { return pool_[e].imag; }

    // SparseMatrix::set_complex: complex values (AC).  Magnitudes become
    // |re| + |im| (element_mag, src/solver/element.hpp:18-20) and the
    // elimination complex_row_col_elimination (src/solver/factor.cpp:769-806).
    void set_complex(bool on) { complex_ = on; }
    bool is_complex() const { return complex_; }

    // NeoSolver::load_real + SparseMatrix::clear_for_load: originals are
    // overwritten by the caller; fill-ins are reset to zero here.
    void clear_fillins();

    // SparseMatrix::mna_preorder (src/solver/utils.cpp:8-89).
    void mna_preorder();

    // SparseMatrix::add_diag_gmin (src/solver/utils.cpp:91-97).
    void add_diag_gmin(double gmin);

    // SparseMatrix::order_and_factor (src/solver/factor.cpp:911-978) with
    // rhs == nullptr, on the currently loaded values.  First call: full
    // Markowitz ordering.  Later calls: re-validate each pivot against the
    // threshold and re-order from the first failing step.
    OrderStatus order_and_factor(double rel_threshold, double abs_threshold,
                                 bool diag_pivoting);

    // --- exports, valid after order_and_factor ---
    int32_t size() const { return size_; }
    int32_t element_count() const { return static_cast<int32_t>(pool_.size()); }
    int32_t fillin_count() const { return fillins_; }
    // First step at which the last re-validation found a failing pivot
    // (0 when no re-ordering happened).
    int32_t reorder_step() const { return reorder_step_; }
    // 1-based: internal index -> external row / column.
    const std::vector<int32_t>& int_to_ext_row() const { return int_to_ext_row_; }
    const std::vector<int32_t>& int_to_ext_col() const { return int_to_ext_col_; }

    // Walk column j (internal, 1-based) top to bottom.
    int32_t first_in_col(int32_t j) const { return first_in_col_[j]; }
    int32_t next_in_col(int32_t e) const { return pool_[e].next_in_col; }
    int32_t row_of(int32_t e) const { return pool_[e].row; }
    int32_t diag(int32_t i) const { return diag_[i]; }
    bool is_fillin(int32_t e) const { return pool_[e].fill; }
    bool ordered() const { return !needs_ordering_; }

private:
    struct Element {
        double val = 0.0;
        double imag = 0.0;
        int32_t row = 0;
        int32_t col = 0;
        int32_t next_in_row = -1;
        int32_t next_in_col = -1;
        bool fill = false;
    };

    int32_t size_;
    int32_t current_size_ = 0;
    bool needs_ordering_ = true;
    bool rows_linked_ = false;
    bool preordered_ = false;
    bool complex_ = false;
    double rel_threshold_ = 1.0e-3;
    double abs_threshold_ = 0.0;
    OrderStatus error_ = OrderStatus::ok;
    int32_t fillins_ = 0;
    int32_t singletons_ = 0;
    int32_t reorder_step_ = 0;

    std::vector<Element> pool_;
    std::vector<int32_t> first_in_col_, first_in_row_, diag_;
    std::vector<int32_t> int_to_ext_row_, int_to_ext_col_;
    std::vector<int32_t> ext_to_int_row_, ext_to_int_col_;
    std::vector<int32_t> mrow_, mcol_;
    std::vector<long> mprod_;
    std::vector<double> work_;

    double mag(int32_t e) const;
    void translate(int32_t& row, int32_t& col);
    int32_t new_element(int32_t row, int32_t col, bool fill);
    void insert_in_col(int32_t e, int32_t col);
    void insert_in_row(int32_t e, int32_t row);
    int32_t find_in_col(int32_t col, int32_t row) const;
    void link_rows();
    int32_t count_twins(int32_t col, int32_t& t1, int32_t& t2);
    void swap_cols(int32_t t1, int32_t t2);

    double largest_in_col_from(int32_t e) const;
    double largest_in_col_excluding(int32_t e, int32_t step) const;
    void count_markowitz(int32_t step);
    void markowitz_products(int32_t step);
    long product_of(int32_t r, int32_t c) const;
    int32_t search_for_pivot(int32_t step, bool diag_pivoting);
    int32_t search_singleton(int32_t step);
    int32_t search_diagonal_quick(int32_t step);
    int32_t search_diagonal_full(int32_t step);
    int32_t search_whole(int32_t step);
    void exchange(int32_t pivot, int32_t step);
    void swap_rows(int32_t r1, int32_t r2);
    void swap_columns(int32_t c1, int32_t c2);
    void eliminate(int32_t pivot);
    void eliminate_complex(int32_t pivot);
    int32_t create_fillin(int32_t row, int32_t col);
    void update_markowitz(int32_t pivot);
};

}  // namespace nsg
