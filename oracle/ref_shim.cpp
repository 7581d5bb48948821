// Test infrastructure only: an extern "C" export shim compiled against the
// reference's own headers and linked with the reference's own sources (see
// oracle/Makefile).  It is the checker for this repository's symbolic phase,
// refactor and solves, and the CPU baseline in bench.py.  Nothing in the
// product (neospice_b200/) links or loads it.
//
// The reference keeps the Sparse-1.3 state of a NeoSolver private
// (src/core/neo_solver.hpp:37-68, src/solver/matrix.hpp:61-175).  The export
// functions below read it by re-opening the access specifiers for this one
// translation unit; the class layout is unchanged.
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <memory>
#include <sstream>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "api/neospice.hpp"
#include "core/circuit.hpp"
#include "core/dc.hpp"
#include "core/matrix.hpp"
#include "core/newton.hpp"
#include "core/solver_iface.hpp"
#include "solver/config.hpp"
#include "solver/error.hpp"
#include "solver/element.hpp"

#define private public
#include "core/neo_solver.hpp"
#include "solver/matrix.hpp"
#undef private

using namespace neospice;

// The reference links LAPACK only for .pz (src/core/pz.cpp:24); the oracle
// never runs .pz, so a stub that reports failure stands in for it.
extern "C" void dggev_(char*, char*, int*, double*, int*, double*, int*,
                       double*, double*, double*, double*, int*, double*,
                       int*, double*, int*, int* info) {
    if (info) *info = -1;
}

namespace {

struct RefSolver {
    int n = 0;
    int nnz = 0;
    SparsityPattern pattern;
    NumericMatrix mat;
    NeoSolver solver;
    RefSolver(int n_, std::vector<std::pair<int32_t, int32_t>> entries)
        : n(n_), nnz(static_cast<int>(entries.size())),
          pattern(n_, std::move(entries)), mat(pattern) {}
};

}  // namespace

extern "C" {

// NeoSolver::symbolic on a CSC pattern (0-based, rows sorted per column).
void* nsref_solver_create(int n, int nnz, const int* col_ptr, const int* row_idx) {
    std::vector<std::pair<int32_t, int32_t>> entries;
    entries.reserve(nnz);
    for (int j = 0; j < n; ++j)
        for (int p = col_ptr[j]; p < col_ptr[j + 1]; ++p)
            entries.emplace_back(row_idx[p], j);
    auto* rs = new RefSolver(n, std::move(entries));
    rs->solver.symbolic(rs->pattern);
    return rs;
}

void nsref_solver_destroy(void* h) { delete static_cast<RefSolver*>(h); }

// NeoSolver::numeric (neo_solver.cpp:219-245): returns 1 when singular,
// -1 when the reference threw.
int nsref_solver_numeric(void* h, const double* values, double diag_gmin) {
    auto* rs = static_cast<RefSolver*>(h);
    std::memcpy(rs->mat.data(), values, sizeof(double) * rs->nnz);
    try {
        return rs->solver.numeric(rs->pattern, rs->mat, diag_gmin) ? 1 : 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// NeoSolver::refactorize (neo_solver.cpp:247-265).
int nsref_solver_refactor(void* h, const double* values, double diag_gmin) {
    auto* rs = static_cast<RefSolver*>(h);
    std::memcpy(rs->mat.data(), values, sizeof(double) * rs->nnz);
    try {
        return rs->solver.refactorize(rs->mat, diag_gmin) ? 1 : 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// NeoSolver::solve (neo_solver.cpp:267-297); rhs in, solution out.
int nsref_solver_solve(void* h, double* rhs) {
    auto* rs = static_cast<RefSolver*>(h);
    std::vector<double> v(rhs, rhs + rs->n);
    try {
        rs->solver.solve(v);
    } catch (const std::exception&) {
        return -1;
    }
    std::memcpy(rhs, v.data(), sizeof(double) * rs->n);
    return 0;
}

// SparseMatrix::solve_transposed (solve.cpp:102-141) on the factored matrix,
// with the same 1-based staging NeoSolver::solve uses.
int nsref_solver_solve_transposed(void* h, double* rhs) {
    auto* rs = static_cast<RefSolver*>(h);
    auto* m = rs->solver.matrix_.get();
    if (!m || !rs->solver.factored_) return -1;
    std::vector<double> b(rs->n + 1, 0.0), x(rs->n + 1, 0.0);
    for (int i = 0; i < rs->n; ++i) b[i + 1] = rhs[i];
    m->solve_transposed(b.data(), x.data());
    for (int i = 0; i < rs->n; ++i) rhs[i] = x[i + 1];
    return 0;
}

// Element count (originals + fill-ins) of the factored matrix.
int nsref_solver_element_count(void* h) {
    auto* m = static_cast<RefSolver*>(h)->solver.matrix_.get();
    int count = 0;
    for (int j = 1; j <= m->size_; ++j)
        for (auto* e = m->first_in_col_[j]; e; e = e->NextInCol) ++count;
    return count;
}

// Export the factored structure: elements enumerated column by column in
// internal (pivot) order, rows ascending.  elem_row/elem_col are internal
// 1-based indices, elem_val the stored factor value (L unscaled, U scaled by
// the reciprocal pivot, pivot stored as its reciprocal), slot_to_elem maps
// each CSC slot of the pattern to its element, int_to_ext_* are 1-based.
int nsref_solver_export(void* h, int* int_to_ext_row, int* int_to_ext_col,
                        int* elem_row, int* elem_col, double* elem_val,
                        int* slot_to_elem) {
    auto* rs = static_cast<RefSolver*>(h);
    auto* m = rs->solver.matrix_.get();
    std::unordered_map<const double*, int> where;
    int e_idx = 0;
    for (int j = 1; j <= m->size_; ++j) {
        for (auto* e = m->first_in_col_[j]; e; e = e->NextInCol) {
            elem_row[e_idx] = e->Row;
            elem_col[e_idx] = j;
            elem_val[e_idx] = e->Real;
            where[&e->Real] = e_idx;
            ++e_idx;
        }
    }
    for (int i = 1; i <= m->size_; ++i) {
        int_to_ext_row[i - 1] = m->int_to_ext_row_[i];
        int_to_ext_col[i - 1] = m->int_to_ext_col_[i];
    }
    for (int k = 0; k < rs->nnz; ++k) {
        auto it = where.find(rs->solver.element_ptrs_[k]);
        slot_to_elem[k] = (it == where.end()) ? -1 : it->second;
    }
    return e_idx;
}

namespace {

// The diode-clamped mesh through the reference's typed Circuit API.  Node
// (x, y) is "n<y*side+x>" and is created in that order, so its MNA index is
// y*side+x; the corner source's branch current follows at index side*side.
// r_h holds the (side-1)*side horizontal resistors (x, y)-(x+1, y) row by
// row, r_v the side*(side-1) vertical ones (x, y)-(x, y+1).  Devices are
// created R (horizontal, then vertical), D, I, V in that order.
void build_mesh(Circuit& ckt, int side, const double* r_h, const double* r_v, int n_diodes,
                const int* diode_node, double is, double n_emis, int n_isrc,
                const int* isrc_node, const double* isrc_amps, double v_corner) {
    const int N = side * side;
    std::vector<NodeId> nodes(N);
    for (int i = 0; i < N; ++i) nodes[i] = ckt.node("n" + std::to_string(i));
    int k = 0;
    for (int y = 0; y < side; ++y)
        for (int x = 0; x + 1 < side; ++x, ++k)
            ckt.R("rh" + std::to_string(k), nodes[y * side + x], nodes[y * side + x + 1], r_h[k]);
    k = 0;
    for (int y = 0; y + 1 < side; ++y)
        for (int x = 0; x < side; ++x, ++k)
            ckt.R("rv" + std::to_string(k), nodes[y * side + x], nodes[(y + 1) * side + x], r_v[k]);
    char card[160];
    std::snprintf(card, sizeof card, ".model dmod D(IS=%.17g N=%.17g)", is, n_emis);
    ckt.model(card);
    for (int d = 0; d < n_diodes; ++d)
        ckt.D("d" + std::to_string(d), nodes[diode_node[d]], GND, "dmod");
    for (int s = 0; s < n_isrc; ++s)
        ckt.I("i" + std::to_string(s), GND, nodes[isrc_node[s]], isrc_amps[s]);
    ckt.V("vc", nodes[0], GND, v_corner);
    ckt.finalize_if_needed();
}

}  // namespace

// DC operating point of the mesh through solve_dc (Simulator::run_dc's
// engine).  Returns the number of unknowns written to solution, or -1 when
// the reference threw.
int nsref_mesh_dc(int side, const double* r_h, const double* r_v, int n_diodes,
                  const int* diode_node, double is, double n_emis, int n_isrc,
                  const int* isrc_node, const double* isrc_amps, double v_corner,
                  double* solution, int* iterations, double* seconds) {
    try {
        auto t0 = std::chrono::steady_clock::now();
        Circuit ckt;
        build_mesh(ckt, side, r_h, r_v, n_diodes, diode_node, is, n_emis, n_isrc, isrc_node,
                   isrc_amps, v_corner);
        DCResult res = solve_dc(ckt);
        const auto* op = ckt.operating_point();
        const int nv = ckt.num_vars();
        if (!op) return -1;
        for (int i = 0; i < nv; ++i) solution[i] = (*op)[i];
        if (iterations) *iterations = res.status.iterations;
        auto t1 = std::chrono::steady_clock::now();
        if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
        return nv;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "nsref_mesh_dc: %s\n", e.what());
        return -1;
    }
}

// The matrix and rhs of the first DC Newton iteration (MODEDCOP |
// MODEINITJCT, zero guess): newton_solve's device-load block
// (src/core/newton.cpp:141-175) run once.  col_ptr (num_vars+1), row_idx
// (nnz), values (nnz), rhs (num_vars).  Returns nnz, or -1.  Call with null
// arrays to get sizes: *num_vars and the return value.
int nsref_mesh_initjct(int side, const double* r_h, const double* r_v, int n_diodes,
                       const int* diode_node, double is, double n_emis, int n_isrc,
                       const int* isrc_node, const double* isrc_amps, double v_corner,
                       int* num_vars, int* col_ptr, int* row_idx, double* values, double* rhs_out) {
    try {
        Circuit ckt;
        build_mesh(ckt, side, r_h, r_v, n_diodes, diode_node, is, n_emis, n_isrc, isrc_node,
                   isrc_amps, v_corner);
        const int n = ckt.num_vars();
        const auto& pattern = ckt.pattern();
        if (num_vars) *num_vars = n;
        if (!col_ptr) return pattern.nnz();
        CSCData csc = pattern.to_csc();
        for (int j = 0; j <= n; ++j) col_ptr[j] = csc.col_ptr[j];
        for (int k = 0; k < pattern.nnz(); ++k) row_idx[k] = csc.row_idx[k];

        ckt.integrator_ctx.options = &ckt.options;
        ckt.integrator_ctx.mode = 0x10 | 0x200;  // MODEDCOP | MODEINITJCT
        NumericMatrix mat(pattern);
        std::vector<double> solution(n, 0.0), rhs(n, 0.0);
        std::vector<double> ob_sol(n + 1, 0.0), ob_rhs(n + 1, 0.0);
        OneBasedEvalArrays arrays{ob_sol.data(), ob_rhs.data(), n + 1};
        tls_integrator_ctx = &ckt.integrator_ctx;
        tls_one_based_eval_arrays = &arrays;
        for (Device* dev : ckt.device_load_order()) dev->evaluate(solution, mat, rhs);
        tls_one_based_eval_arrays = nullptr;
        tls_integrator_ctx = nullptr;
        for (int i = 0; i < n; ++i) rhs[i] += ob_rhs[i + 1];
        const double pin = (ckt.options.gmin > 0.0) ? ckt.options.gmin : 1e-12;
        for (int32_t idx : ckt.dead_node_indices()) mat.add(pattern.offset(idx, idx), pin);
        for (int k = 0; k < pattern.nnz(); ++k) values[k] = mat.data()[k];
        for (int i = 0; i < n; ++i) rhs_out[i] = rhs[i];
        return pattern.nnz();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "nsref_mesh_initjct: %s\n", e.what());
        return -1;
    }
}

}  // extern "C"
