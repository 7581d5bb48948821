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
#include <cstdlib>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "api/neospice.hpp"
#include "core/circuit.hpp"
#include "core/dc.hpp"
#include "core/transient.hpp"
#include "core/sens.hpp"
#include "devices/capacitor.hpp"
#include "devices/isource.hpp"
#include "devices/vsource.hpp"
#include "core/matrix.hpp"
#include "core/newton.hpp"
#include "core/solver_iface.hpp"
#include "solver/config.hpp"
#include "solver/error.hpp"
#include "solver/element.hpp"

#include "core/amd.hpp"
#include "core/convergence.hpp"

#define private public
#include "devices/bsim4v7/bsim4v7_device.hpp"
#include "core/neo_solver.hpp"
#include "core/amd_lu_solver.hpp"
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

// ---- complex (AC) path of NeoSolver (src/core/neo_solver.cpp:104-111,
// 228-284) ------------------------------------------------------------------

// NeoSolver::numeric_complex on interleaved (re, im) values, 2*nnz doubles.
int nsref_solver_numeric_complex(void* h, const double* ax) {
    auto* rs = static_cast<RefSolver*>(h);
    try {
        rs->solver.numeric_complex(rs->pattern, std::vector<double>(ax, ax + 2 * rs->nnz));
    } catch (const std::exception&) {
        return -1;
    }
    return 0;
}

// NeoSolver::refactorize_complex: 1 when singular.
int nsref_solver_refactor_complex(void* h, const double* ax) {
    auto* rs = static_cast<RefSolver*>(h);
    try {
        return rs->solver.refactorize_complex(std::vector<double>(ax, ax + 2 * rs->nnz)) ? 1 : 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// NeoSolver::solve_complex: rhs (2*n interleaved) in, solution out.
int nsref_solver_solve_complex(void* h, double* rhs) {
    auto* rs = static_cast<RefSolver*>(h);
    std::vector<double> v(rhs, rhs + 2 * rs->n);
    try {
        rs->solver.solve_complex(v);
    } catch (const std::exception&) {
        return -1;
    }
    std::memcpy(rhs, v.data(), sizeof(double) * 2 * rs->n);
    return 0;
}

// The imaginary parts of the factored elements, in nsref_solver_export's
// element order.
int nsref_solver_export_imag(void* h, double* elem_imag) {
    auto* m = static_cast<RefSolver*>(h)->solver.matrix_.get();
    int e_idx = 0;
    for (int j = 1; j <= m->size_; ++j)
        for (auto* e = m->first_in_col_[j]; e; e = e->NextInCol) elem_imag[e_idx++] = e->Imag;
    return e_idx;
}

// ---- AMD-LU (src/core/amd.cpp, src/core/amd_lu_solver.cpp) ----------------

// amd_ordering on a CSC pattern; perm receives n entries.
int nsref_amd_order(int n, const int* col_ptr, const int* row_idx, int* perm) {
    auto q = amd_ordering(n, col_ptr, row_idx);
    for (size_t k = 0; k < q.size(); ++k) perm[k] = q[k];
    return static_cast<int>(q.size());
}

namespace {
struct RefAmd {
    int n = 0;
    int nnz = 0;
    SparsityPattern pattern;
    NumericMatrix mat;
    AmdLuSolver solver;
    RefAmd(int n_, std::vector<std::pair<int32_t, int32_t>> entries)
        : n(n_), nnz(static_cast<int>(entries.size())),
          pattern(n_, std::move(entries)), mat(pattern) {}
};
}  // namespace

// AmdLuSolver::symbolic on a CSC pattern (0-based, rows sorted per column).
void* nsref_amdlu_create(int n, int nnz, const int* col_ptr, const int* row_idx) {
    std::vector<std::pair<int32_t, int32_t>> entries;
    entries.reserve(nnz);
    for (int j = 0; j < n; ++j)
        for (int p = col_ptr[j]; p < col_ptr[j + 1]; ++p) entries.emplace_back(row_idx[p], j);
    auto* ra = new RefAmd(n, std::move(entries));
    ra->solver.symbolic(ra->pattern);
    return ra;
}

void nsref_amdlu_destroy(void* h) { delete static_cast<RefAmd*>(h); }

// AmdLuSolver::numeric: 1 when singular, -1 when the reference threw.
int nsref_amdlu_numeric(void* h, const double* values, double diag_gmin) {
    auto* ra = static_cast<RefAmd*>(h);
    std::memcpy(ra->mat.data(), values, sizeof(double) * ra->nnz);
    try {
        return ra->solver.numeric(ra->pattern, ra->mat, diag_gmin) ? 1 : 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// AmdLuSolver::refactorize (replay, full factor_ on a failed growth test).
int nsref_amdlu_refactor(void* h, const double* values, double diag_gmin) {
    auto* ra = static_cast<RefAmd*>(h);
    std::memcpy(ra->mat.data(), values, sizeof(double) * ra->nnz);
    try {
        return ra->solver.refactorize(ra->mat, diag_gmin) ? 1 : 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// Replay / fallback counters of refactorize().
void nsref_amdlu_counts(void* h, int* fast, int* fallback) {
    auto* ra = static_cast<RefAmd*>(h);
    *fast = ra->solver.refactor_fast_count();
    *fallback = ra->solver.refactor_fallback_count();
}

int nsref_amdlu_solve(void* h, double* rhs) {
    auto* ra = static_cast<RefAmd*>(h);
    std::vector<double> v(rhs, rhs + ra->n);
    try {
        ra->solver.solve(v);
    } catch (const std::exception&) {
        return -1;
    }
    std::memcpy(rhs, v.data(), sizeof(double) * ra->n);
    return 0;
}

// Sizes of L and U (entries incl. the diagonals).
void nsref_amdlu_sizes(void* h, int* nnz_l, int* nnz_u) {
    auto* ra = static_cast<RefAmd*>(h);
    *nnz_l = static_cast<int>(ra->solver.Li_.size());
    *nnz_u = static_cast<int>(ra->solver.Ui_.size());
}

// The factor as AmdLuSolver stores it: q (n), pinv (n), Lp/Up (n+1),
// Li/Lx (nnz_l), Ui/Ux (nnz_u); L rows in pivot-step space.
void nsref_amdlu_export(void* h, int* q, int* pinv, int* Lp, int* Li, double* Lx, int* Up,
                        int* Ui, double* Ux) {
    auto& s = static_cast<RefAmd*>(h)->solver;
    std::copy(s.q_.begin(), s.q_.end(), q);
    std::copy(s.pinv_.begin(), s.pinv_.end(), pinv);
    std::copy(s.Lp_.begin(), s.Lp_.end(), Lp);
    std::copy(s.Li_.begin(), s.Li_.end(), Li);
    std::copy(s.Lx_.begin(), s.Lx_.end(), Lx);
    std::copy(s.Up_.begin(), s.Up_.end(), Up);
    std::copy(s.Ui_.begin(), s.Ui_.end(), Ui);
    std::copy(s.Ux_.begin(), s.Ux_.end(), Ux);
}

// make_solver(num_vars, is_linear)->name() under the current environment.
int nsref_make_solver_name(int num_vars, int is_linear, char* out, int cap) {
    auto s = make_solver(num_vars, is_linear != 0);
    std::snprintf(out, cap, "%s", s->name());
    return 0;
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

// ---------------------------------------------------------------------------
// Generic runner on a line-based circuit description, built through the
// reference's typed Circuit API in the order given (so node numbering and
// device load order match a circuit built the same way elsewhere):
//   nodes N                          nodes n0..n{N-1} (MNA indices 0..N-1)
//   R a b ohms | C a b farads [ic] | V a b dc | I a b dc
//   VPULSE a b v1 v2 td tr tf pw per | IPULSE ... | VPWL a b t0 v0 t1 v1 ...
//   IPWL a b t0 v0 ... | D a k IS N | MODEL name card... | M d g s b model W L [DELVTO]
//   OPT name value                   (reltol, abstol, vntol, gmin, itl4, method, temp)
// Node -1 is ground.  analysis 0 = DC operating point, 1 = transient.
struct SimResult {
    std::string error;
    int num_nodes = 0, num_vars = 0, iterations = 0, rejected = 0, method = 0;
    double seconds = 0.0;
    std::vector<double> times;
    std::vector<double> values;  // npoints x (num_vars for DC, num_nodes for tran)
};

static NodeId node_of(const std::vector<NodeId>& nodes, int k) {
    return k < 0 ? GND : nodes.at(k);
}

// Build a circuit from a description (format above) through the typed API.
static void build_from_desc(Circuit& ckt, const char* desc) {
    // Tokenised by hand (strtod/strtol): iostreams are avoided because
    // the loading process may carry a different C++ runtime.
    std::vector<std::vector<std::string>> lines;
    {
        std::vector<std::string> cur;
        std::string tok;
        for (const char* p = desc;; ++p) {
            const char c = *p;
            if (c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\0') {
                if (!tok.empty()) cur.push_back(tok), tok.clear();
                if ((c == '\n' || c == '\0') && !cur.empty()) lines.push_back(cur), cur.clear();
                if (c == '\0') break;
            } else {
                tok.push_back(c);
            }
        }
    }
    std::vector<NodeId> nodes;
    int dev = 0;
    for (const auto& tk : lines) {
        const std::string& kind = tk[0];
        const std::string name = kind + std::to_string(dev++);
        auto I_ = [&](size_t k) { return static_cast<int>(std::strtol(tk.at(k).c_str(), nullptr, 10)); };
        auto D_ = [&](size_t k) { return std::strtod(tk.at(k).c_str(), nullptr); };
        auto rest = [&](size_t from) {
            std::vector<double> v;
            for (size_t k = from; k < tk.size(); ++k) v.push_back(D_(k));
            return v;
        };
        if (kind == "nodes") {
            const int n = I_(1);
            for (int i = 0; i < n; ++i) nodes.push_back(ckt.node("n" + std::to_string(i)));
        } else if (kind == "R" || kind == "C" || kind == "V" || kind == "I") {
            NodeId a = node_of(nodes, I_(1)), b = node_of(nodes, I_(2));
            auto v = rest(3);
            if (kind == "R") ckt.R(name, a, b, v.at(0));
            else if (kind == "C") {
                if (v.size() > 1) ckt.C(name, a, b, v[0], v[1]);
                else ckt.C(name, a, b, v.at(0));
            } else if (kind == "V") ckt.V(name, a, b, v.at(0));
            else ckt.I(name, a, b, v.at(0));
        } else if (kind == "VPULSE" || kind == "IPULSE" || kind == "VPWL" || kind == "IPWL") {
            NodeId a = node_of(nodes, I_(1)), b = node_of(nodes, I_(2));
            auto v = rest(3);
            const bool is_v = kind[0] == 'V';
            DevId id = is_v ? ckt.V(name, a, b, 0.0) : ckt.I(name, a, b, 0.0);
            Device* d = ckt.devices()[static_cast<int32_t>(id)].get();
            if (kind == "VPULSE" || kind == "IPULSE") {
                PulseParams pp{v.at(0), v.at(1), v.at(2), v.at(3), v.at(4), v.at(5), v.at(6)};
                if (is_v) static_cast<VSource*>(d)->set_pulse(pp);
                else static_cast<ISource*>(d)->set_pulse(pp);
            } else {
                PwlParams pw;
                for (size_t k = 0; k + 1 < v.size(); k += 2) pw.points.emplace_back(v[k], v[k + 1]);
                if (is_v) static_cast<VSource*>(d)->set_pwl(pw);
                else static_cast<ISource*>(d)->set_pwl(pw);
            }
        } else if (kind == "D") {
            // D a k IS N [CJO VJ M FC TT [BV IBV NBV [RS]]]; BV nan: not given
            char card[400];
            if (tk.size() > 10) {
                int w = std::snprintf(card, sizeof card,
                                      ".model dm%d D(IS=%.17g N=%.17g CJO=%.17g VJ=%.17g M=%.17g "
                                      "FC=%.17g TT=%.17g",
                                      dev, D_(3), D_(4), D_(5), D_(6), D_(7), D_(8), D_(9));
                if (!std::isnan(D_(10)))
                    w += std::snprintf(card + w, sizeof card - w, " BV=%.17g IBV=%.17g NBV=%.17g",
                                       D_(10), D_(11), D_(12));
                if (tk.size() > 13 && D_(13) != 0.0)
                    w += std::snprintf(card + w, sizeof card - w, " RS=%.17g", D_(13));
                std::snprintf(card + w, sizeof card - w, ")");
            } else if (tk.size() > 5)
                std::snprintf(card, sizeof card,
                              ".model dm%d D(IS=%.17g N=%.17g CJO=%.17g VJ=%.17g M=%.17g FC=%.17g "
                              "TT=%.17g)",
                              dev, D_(3), D_(4), D_(5), D_(6), D_(7), D_(8), D_(9));
            else
                std::snprintf(card, sizeof card, ".model dm%d D(IS=%.17g N=%.17g)", dev, D_(3), D_(4));
            ckt.model(card);
            ckt.D(name, node_of(nodes, I_(1)), node_of(nodes, I_(2)), "dm" + std::to_string(dev));
        } else if (kind == "MODEL") {
            std::string card;
            for (size_t k = 1; k < tk.size(); ++k) card += (k > 1 ? " " : "") + tk[k];
            ckt.model(card);
        } else if (kind == "M") {
            DevId id = ckt.M(name, node_of(nodes, I_(1)), node_of(nodes, I_(2)),
                             node_of(nodes, I_(3)), node_of(nodes, I_(4)), tk.at(5), D_(6), D_(7));
            if (tk.size() > 8) {  // DELVTO of a BSIM4v7 instance (bsim4v7_param.cpp:142-144)
                auto* b4 = dynamic_cast<BSIM4v7Device*>(ckt.devices()[static_cast<int32_t>(id)].get());
                if (!b4) throw std::invalid_argument("delvto given for a non-BSIM4v7 MOSFET");
                b4->inst_.BSIM4v7delvto = D_(8);
                b4->inst_.BSIM4v7delvtoGiven = 1;
            }
        } else if (kind == "OPT") {
            const std::string& key = tk.at(1);
            const double val = D_(2);
            if (key == "reltol") ckt.options.reltol = val;
            else if (key == "abstol") ckt.options.abstol = val;
            else if (key == "vntol") ckt.options.vntol = val;
            else if (key == "gmin") ckt.options.gmin = val;
            else if (key == "itl4") ckt.options.itl4 = static_cast<int>(val);
            else if (key == "gear") ckt.options.method = val != 0.0 ? "gear" : "trap";
            else if (key == "verbose") ckt.options.verbose = val != 0.0;
            else if (key == "temp") ckt.options.temp = val;  // kelvin
        } else {
            throw std::invalid_argument("unknown line kind: " + kind);
        }
    }
    ckt.finalize_if_needed();
}

void* nsref_sim_run(const char* desc, int analysis, double tstep, double tstop) {
    auto* res = new SimResult;
    try {
        auto t0 = std::chrono::steady_clock::now();
        Circuit ckt;
        build_from_desc(ckt, desc);
        res->num_nodes = ckt.num_nodes();
        res->num_vars = ckt.num_vars();
        if (analysis == 2 || analysis == 3 || analysis == 4) {
            // The reference's source_stepping (2), gain_stepping (3) or
            // pseudo_transient (4) run directly, set up as solve_dc sets up
            // its cascade (dc.cpp:80-96, 176-224): solver, symbolic, options
            // published, MODEDCOP | MODEINITJCT, zero guess.
            const int32_t n = ckt.num_vars();
            std::vector<double> solution(n, 0.0);
            auto solver = make_solver(n, ckt.is_linear());
            solver->symbolic(ckt.pattern());
            ckt.integrator_ctx.options = &ckt.options;
            ckt.integrator_ctx.mode = 0x10 | 0x200;
            NewtonResult r =
                analysis == 2 ? source_stepping(ckt, *solver, solution, ckt.options)
                : analysis == 3 ? gain_stepping(ckt, *solver, solution, ckt.options)
                                : pseudo_transient(ckt, *solver, solution, ckt.options);
            res->times.push_back(0.0);
            res->values = solution;
            res->iterations = r.iterations;
            res->method = r.converged ? (analysis == 4 ? 3 : 2) : -1;
        } else if (analysis == 0) {
            DCResult r = solve_dc(ckt);
            const auto* op = ckt.operating_point();
            if (!op) throw std::runtime_error("no operating point");
            res->times.push_back(0.0);
            res->values.assign(op->begin(), op->end());
            res->iterations = r.status.iterations;
            res->method = static_cast<int>(r.status.convergence_method);
        } else {
            TransientResult r = solve_transient(ckt, tstep, tstop);
            res->times = r.time;
            const size_t np = r.time.size();
            res->values.resize(np * res->num_nodes);
            for (int i = 0; i < res->num_nodes; ++i)
                for (size_t k = 0; k < np; ++k) res->values[k * res->num_nodes + i] = r.voltages_dense[i][k];
            res->iterations = r.status.iterations;
            res->rejected = r.rejected_steps;
        }
        res->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    } catch (const std::exception& e) {
        res->error = e.what();
    }
    return res;
}

int nsref_sim_info(void* h, int* num_nodes, int* num_vars, int* npoints, int* iterations,
                   double* seconds, int* rejected) {
    auto* r = static_cast<SimResult*>(h);
    if (num_nodes) *num_nodes = r->num_nodes;
    if (num_vars) *num_vars = r->num_vars;
    if (npoints) *npoints = static_cast<int>(r->times.size());
    if (iterations) *iterations = r->iterations;
    if (seconds) *seconds = r->seconds;
    if (rejected) *rejected = r->rejected;
    return r->error.empty() ? 0 : -1;
}

int nsref_sim_copy(void* h, double* times, double* values) {
    auto* r = static_cast<SimResult*>(h);
    std::memcpy(times, r->times.data(), sizeof(double) * r->times.size());
    std::memcpy(values, r->values.data(), sizeof(double) * r->values.size());
    return 0;
}

const char* nsref_sim_error(void* h) { return static_cast<SimResult*>(h)->error.c_str(); }

void nsref_sim_free(void* h) { delete static_cast<SimResult*>(h); }

}  // extern "C"

// Simulator::run_step_sweep (src/api/neospice.cpp:228-331) on a described
// circuit with `.op` and `.step <source> start stop step`: the source is the
// description's device line `device` (named as build_from_desc names it).
// Writes up to cap step values, each step's node voltages (num_nodes each)
// and Newton iterations; returns the step count, or -1.
extern "C" int nsref_step_dc(const char* desc, int device, double start, double stop, double step,
                             int cap, double* values, double* volts, int* iterations) {
    try {
        Circuit ckt;
        build_from_desc(ckt, desc);
        std::string name;
        {
            // the device line's kind token, as build_from_desc names devices
            int line = 0;
            const char* p = desc;
            while (*p && line < device) {
                if (*p == '\n') ++line;
                ++p;
            }
            std::string kind;
            while (*p && *p != ' ' && *p != '\n') kind.push_back(*p++);
            name = kind + std::to_string(device);
        }
        StepCommand sc;
        sc.kind = StepCommand::SOURCE;
        sc.name = name;
        sc.start = start;
        sc.stop = stop;
        sc.step = step;
        ckt.step_commands.push_back(sc);
        ckt.analyses.push_back(AnalysisCommand{OpCmd{}});
        Simulator sim;
        SimulationResult r = sim.run(ckt);
        if (!r.step) return -1;
        const int nsteps = static_cast<int>(r.step->step_values.size());
        const int nn = ckt.num_nodes();
        for (int k = 0; k < nsteps && k < cap; ++k) {
            values[k] = r.step->step_values[k];
            const auto& dc = std::get<DCResult>(r.step->results[k].analysis);
            for (int i = 0; i < nn; ++i) volts[static_cast<size_t>(k) * nn + i] = dc.node_voltages_dense.at(i);
            iterations[k] = dc.status.iterations;
        }
        return nsteps;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "nsref_step_dc: %s\n", e.what());
        return -1;
    }
}

// As nsref_step_dc with `.tran tstep tstop` instead of `.op`: per step the
// number of timepoints (counts), then all steps' times and node voltages
// (points x num_nodes) concatenated, at most cap_points points in all.
extern "C" int nsref_step_tran(const char* desc, int device, double start, double stop,
                               double step, double tstep, double tstop, int cap_steps,
                               int cap_points, int* counts, double* times, double* volts,
                               int* iterations) {
    try {
        Circuit ckt;
        build_from_desc(ckt, desc);
        std::string name;
        {
            int line = 0;
            const char* p = desc;
            while (*p && line < device) {
                if (*p == '\n') ++line;
                ++p;
            }
            std::string kind;
            while (*p && *p != ' ' && *p != '\n') kind.push_back(*p++);
            name = kind + std::to_string(device);
        }
        StepCommand sc;
        sc.kind = StepCommand::SOURCE;
        sc.name = name;
        sc.start = start;
        sc.stop = stop;
        sc.step = step;
        ckt.step_commands.push_back(sc);
        TranCmd tc;
        tc.tstep = tstep;
        tc.tstop = tstop;
        ckt.analyses.push_back(AnalysisCommand{tc});
        Simulator sim;
        SimulationResult r = sim.run(ckt);
        if (!r.step) return -1;
        const int nsteps = static_cast<int>(r.step->step_values.size());
        const int nn = ckt.num_nodes();
        int at = 0;
        for (int k = 0; k < nsteps && k < cap_steps; ++k) {
            const auto& tr = std::get<TransientResult>(r.step->results[k].analysis);
            const int np = static_cast<int>(tr.time.size());
            counts[k] = np;
            iterations[k] = tr.status.iterations;
            for (int t = 0; t < np && at < cap_points; ++t, ++at) {
                times[at] = tr.time[t];
                for (int i = 0; i < nn; ++i)
                    volts[static_cast<size_t>(at) * nn + i] = tr.voltages_dense[i][t];
            }
        }
        return nsteps;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "nsref_step_tran: %s\n", e.what());
        return -1;
    }
}

// The matrix and rhs of the first DC Newton iteration of a described circuit
// (as nsref_mesh_initjct).  Returns nnz, or -1.
extern "C" int nsref_sim_initjct(const char* desc, int* num_vars, int* col_ptr, int* row_idx,
                                 double* values, double* rhs_out) {
    try {
        Circuit ckt;
        build_from_desc(ckt, desc);
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
        std::fprintf(stderr, "nsref_sim_initjct: %s\n", e.what());
        return -1;
    }
}

// A sequence of device evaluations of a described circuit, as Newton
// iterations would run them (Device::evaluate of every device in load
// order, UCB rhs folded in), for comparing device loads on the CPU.  Step s
// first applies state_op[s] (0 nothing, 1 rotate_state (circuit.cpp:328),
// 2 copy state0 into state1..3 as the transient's seeding does,
// transient.cpp:790-800), then evaluates at the guess xs + s*n in CKTmode
// modes[s] with ctx + 8*s = {ag0, ag1, ag2, xmu_ratio, delta, delta_old1,
// time, order + 10 * method}; values / rhs receive the matrix (slot order)
// and rhs of each step.  Returns nnz, or -1.
extern "C" int nsref_sim_eval_seq(const char* desc, int nsteps, const int* state_op,
                                  const int* modes, const double* xs, const double* ctx,
                                  double* values, double* rhs_out) {
    try {
        Circuit ckt;
        build_from_desc(ckt, desc);
        const int n = ckt.num_vars();
        const auto& pattern = ckt.pattern();
        const int ns = ckt.num_states();
        ckt.integrator_ctx.options = &ckt.options;
        for (int s = 0; s < nsteps; ++s) {
            if (state_op[s] == 1) {
                ckt.rotate_state();
            } else if (state_op[s] == 2) {
                std::copy_n(ckt.state0(), ns, ckt.state1());
                std::copy_n(ckt.state0(), ns, ckt.state2());
                std::copy_n(ckt.state0(), ns, ckt.state3());
            }
            const double* c = ctx + 8 * s;
            IntegratorCtx& ic = ckt.integrator_ctx;
            ic.mode = modes[s];
            ic.ag[0] = c[0];
            ic.ag[1] = c[1];
            ic.ag[2] = c[2];
            ic.xmu_ratio = c[3];
            ic.delta = c[4];
            ic.delta_old[0] = c[4];
            ic.delta_old[1] = c[5];
            ic.current_time = c[6];
            for (auto& dev : ckt.devices()) {  // update_source_time (transient.cpp:383-393)
                if (auto* vs = dynamic_cast<VSource*>(dev.get())) vs->set_time(c[6]);
                else if (auto* is = dynamic_cast<ISource*>(dev.get())) is->set_time(c[6]);
            }
            ic.order = static_cast<int>(c[7]) % 10;
            ic.integrate_method = static_cast<int>(c[7]) / 10;
            NumericMatrix mat(pattern);
            std::vector<double> solution(xs + static_cast<size_t>(s) * n,
                                         xs + static_cast<size_t>(s + 1) * n);
            std::vector<double> rhs(n, 0.0);
            std::vector<double> ob_sol(n + 1, 0.0), ob_rhs(n + 1, 0.0);
            for (int i = 0; i < n; ++i) ob_sol[i + 1] = solution[i];
            OneBasedEvalArrays arrays{ob_sol.data(), ob_rhs.data(), n + 1};
            tls_integrator_ctx = &ckt.integrator_ctx;
            tls_one_based_eval_arrays = &arrays;
            for (Device* dev : ckt.device_load_order()) dev->evaluate(solution, mat, rhs);
            tls_one_based_eval_arrays = nullptr;
            tls_integrator_ctx = nullptr;
            for (int i = 0; i < n; ++i) rhs[i] += ob_rhs[i + 1];
            for (int k = 0; k < pattern.nnz(); ++k)
                values[static_cast<size_t>(s) * pattern.nnz() + k] = mat.data()[k];
            for (int i = 0; i < n; ++i) rhs_out[static_cast<size_t>(s) * n + i] = rhs[i];
        }
        return pattern.nnz();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "nsref_sim_eval_seq: %s\n", e.what());
        tls_one_based_eval_arrays = nullptr;
        tls_integrator_ctx = nullptr;
        return -1;
    }
}

// The DC convergence method of a finished run (ConvergenceMethod as an int:
// 0 = the direct Newton attempt, 1 = gmin stepping).
extern "C" int nsref_sim_method(void* h) { return static_cast<SimResult*>(h)->method; }

// The reference's DC sensitivity analysis (solve_sens, src/core/sens.cpp:57-140)
// of v(n<output_node>) for a described circuit: entries in the reference's
// order (resistors, then voltage sources, then current sources, each in
// creation order).  Returns the entry count (sens may be NULL to ask), or -1.
extern "C" int nsref_sim_sens(const char* desc, int output_node, double* sens, double* out_value) {
    try {
        Circuit ckt;
        build_from_desc(ckt, desc);
        SensResult r = solve_sens(ckt, "v(n" + std::to_string(output_node) + ")");
        if (out_value) *out_value = r.output_value;
        if (sens)
            for (size_t k = 0; k < r.entries.size(); ++k) sens[k] = r.entries[k].sensitivity;
        return static_cast<int>(r.entries.size());
    } catch (const std::exception& e) {
        std::fprintf(stderr, "nsref_sim_sens: %s\n", e.what());
        return -1;
    }
}
