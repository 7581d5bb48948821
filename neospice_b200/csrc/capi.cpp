// C ABI of libnsgpu (declared in include/nsgpu.h): host symbolic phase, batch
// set-up and the launches of the batched refactor and sweeps.
#include "capi_internal.hpp"
#include "kernels/dc_device.cuh"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace nsg {
cudaError_t launch_refactor(const PlanDesc* plans, const int32_t* pool, const InstDesc* insts,
                            int count, const double* A, double* LU, double diag_gmin,
                            int check_pivots, double rel_threshold, int32_t* status,
                            int32_t* fail_step, int max_col, int max_n, bool allow_flow,
                            double* lrows, double* urows, cudaStream_t stream);
cudaError_t launch_solve(const PlanDesc* plans, const int32_t* pool, const InstDesc* insts,
                         int count, const double* LU, double* X, double* W, bool transposed,
                         const double* lrows, const double* urows, int max_n,
                         cudaStream_t stream);
size_t grid_scratch_bytes(int max_n);
cudaError_t launch_grid_refactor(const PlanDesc* plans, const int32_t* pool,
                                 const InstDesc* insts, int count, const int32_t* n_of,
                                 const double* A, double* LU, double diag_gmin, int check_pivots,
                                 double rel_threshold, int32_t* status, int32_t* fail_step,
                                 double* lrows, double* urows, void* scratch, int colbuf,
                                 int max_col, int32_t* rmaps, int64_t rmap_words,
                                 const int32_t* cta_from_of, cudaStream_t stream);
int64_t grid_rmap_words(int colbuf, int max_col, int max_n);
cudaError_t launch_complex_refactor(const PlanDesc* plans, const int32_t* pool,
                                    const InstDesc* insts, int count, int max_n, const double* A,
                                    double* LU, int32_t* status, cudaStream_t stream);
cudaError_t launch_complex_solve(const PlanDesc* plans, const int32_t* pool, const InstDesc* insts,
                                 int count, const double* LU, double* X, double* W,
                                 cudaStream_t stream);
size_t complex_refactor_smem(int max_n);
cudaError_t launch_grid_solve(const PlanDesc* plans, const int32_t* pool, const InstDesc* insts,
                              int count, const int32_t* n_of, const double* LU,
                              const double* lrows, const double* urows, double* X, double* W,
                              void* scratch, cudaStream_t stream);
}  // namespace nsg

namespace nsg {

// Setters of every translation unit's copy of the bounded-wait limit
// (c_wait_limit, kernels/lu_cta.cuh), registered at library load.
static std::vector<cudaError_t (*)(int)>& wait_limit_setters() {
    static std::vector<cudaError_t (*)(int)> v;
    return v;
}

bool register_wait_limit_setter(cudaError_t (*set)(int polls)) {
    wait_limit_setters().push_back(set);
    return true;
}

}  // namespace nsg

namespace nsg_internal {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

void clear_error() { g_last_error.clear(); }

int cuda_fail(const char* where, cudaError_t e) {
    return fail(e == cudaErrorMemoryAllocation ? NSG_ERR_NOMEM : NSG_ERR_CUDA,
                std::string(where) + ": " + cudaGetErrorString(e));
}

namespace {
// A 0-based CSC pattern with monotone column pointers and sorted, unique,
// in-range rows.
bool valid_csc(int n, const int* col_ptr, const int* row_idx) {
    for (int j = 0; j < n; ++j) {
        if (col_ptr[j + 1] < col_ptr[j]) return false;
        for (int p = col_ptr[j]; p < col_ptr[j + 1]; ++p)
            if (row_idx[p] < 0 || row_idx[p] >= n || (p > col_ptr[j] && row_idx[p] <= row_idx[p - 1]))
                return false;
    }
    return true;
}

// NeoSolver::symbolic on a valid CSC pattern: one engine element per slot.
void make_markowitz(nsg_topology& t, int n, const int* col_ptr, const int* row_idx) {
    t.engine = std::make_unique<nsg::MarkowitzOrder>(n);
    t.slot_elem.assign(col_ptr[n], 0);
    for (int j = 0; j < n; ++j)
        for (int p = col_ptr[j]; p < col_ptr[j + 1]; ++p)
            t.slot_elem[p] = t.engine->get_element(row_idx[p] + 1, j + 1);
}
}  // namespace

int select_solver(int num_vars, bool is_linear) {
    // read_choice (make_solver.cpp:41-55): NEOSPICE_SOLVER first, then the
    // legacy NEOSPICE_FORCE_AMDLU alias.
    if (const char* s = std::getenv("NEOSPICE_SOLVER")) {
        if (std::strcmp(s, "amdlu") == 0 || std::strcmp(s, "klu") == 0) return NSG_SOLVER_AMDLU;
        if (std::strcmp(s, "markowitz") == 0 || std::strcmp(s, "sparse") == 0)
            return NSG_SOLVER_MARKOWITZ;
    }
    if (const char* f = std::getenv("NEOSPICE_FORCE_AMDLU"))
        if (f[0] != '\0' && std::strcmp(f, "0") != 0) return NSG_SOLVER_AMDLU;
    // Auto: AMD-LU (with the Markowitz fallback) for linear circuits of at
    // least 256 unknowns (kAmdLuAutoThreshold).
    return (num_vars >= 256 && is_linear) ? NSG_SOLVER_AUTO_AMDLU : NSG_SOLVER_MARKOWITZ;
}

void rebuild_plan(nsg_topology& t) {
    t.plan = t.amd ? nsg::build_plan_amd(*t.amd) : nsg::build_plan(*t.engine, t.slot_elem);
}

// numeric() on the host engine.  Markowitz: NeoSolver::numeric's load +
// preorder + gmin + order_and_factor (neo_solver.cpp:219-245).  AMD-LU:
// AmdLuSolver::numeric = factor_ (amd_lu_solver.cpp:273-278), wrapped by
// AutoFallbackSolver::numeric (make_solver.cpp:85-101) when auto-selected.
int numeric_on_engine(nsg_topology& t, const double* values, double diag_gmin) {
    if (t.amd) {
        const bool ok = t.amd->factor(values, diag_gmin);
        if (!ok && t.auto_fallback && !t.committed) {
            const auto& f = *t.amd;
            make_markowitz(t, f.size(), f.col_ptr().data(), f.row_idx().data());
            t.amd.reset();
            t.committed = true;
            return numeric_on_engine(t, values, diag_gmin);
        }
        t.committed = true;
        return ok ? NSG_OK : NSG_SINGULAR;
    }
    t.committed = true;
    auto& mo = *t.engine;
    mo.clear_fillins();
    for (size_t k = 0; k < t.slot_elem.size(); ++k) mo.value(t.slot_elem[k]) = values[k];
    mo.mna_preorder();
    mo.add_diag_gmin(diag_gmin);
    const nsg::OrderStatus st = mo.order_and_factor(1e-3, 1e-13, true);
    if (st == nsg::OrderStatus::no_memory) return NSG_ERR_NOMEM;
    if (st == nsg::OrderStatus::singular) return NSG_SINGULAR;
    return NSG_OK;
}

int order_topology(int n, int nnz, const int* col_ptr, const int* row_idx, const double* values,
                   double diag_gmin, std::unique_ptr<nsg_topology>& out, int solver) {
    if (n <= 0 || nnz <= 0 || !col_ptr || !row_idx || !values)
        return fail(NSG_ERR_INVALID, "nsg_topology_order: bad arguments");
    if (col_ptr[0] != 0 || col_ptr[n] != nnz)
        return fail(NSG_ERR_INVALID, "nsg_topology_order: col_ptr does not span nnz");
    if (solver != NSG_SOLVER_MARKOWITZ && solver != NSG_SOLVER_AMDLU &&
        solver != NSG_SOLVER_AUTO_AMDLU)
        return fail(NSG_ERR_INVALID, "nsg_topology_order: unknown solver");
    if (!valid_csc(n, col_ptr, row_idx))
        return fail(NSG_ERR_INVALID, "nsg_topology_order: col_ptr not monotone or rows not "
                                     "sorted/unique");
    auto t = std::make_unique<nsg_topology>();
    if (solver == NSG_SOLVER_MARKOWITZ) {
        make_markowitz(*t, n, col_ptr, row_idx);
    } else {
        // AmdLuSolver::symbolic: the AMD order of the pattern.
        t->amd = std::make_unique<nsg::AmdLuFactor>(
            n, std::vector<int32_t>(col_ptr, col_ptr + n + 1),
            std::vector<int32_t>(row_idx, row_idx + nnz));
        t->auto_fallback = (solver == NSG_SOLVER_AUTO_AMDLU);
    }
    const int rc = numeric_on_engine(*t, values, diag_gmin);
    if (rc == NSG_SINGULAR) return fail(NSG_SINGULAR, "nsg_topology_order: singular matrix");
    if (rc != NSG_OK) return fail(rc, "nsg_topology_order: ordering failed");
    rebuild_plan(*t);
    out = std::move(t);
    return NSG_OK;
}

nsg::PlanDesc make_plan_desc(const nsg::TopologyPlan& p, std::vector<int32_t>& pool) {
    nsg::PlanDesc d{};
    d.n = p.n;
    d.nnz_a = p.nnz_a;
    d.nnz_lu = p.nnz_lu;
    d.n_col_lev = static_cast<int32_t>(p.col_lev_ptr.size()) - 1;
    d.n_fwd_lev = static_cast<int32_t>(p.fwd_lev_ptr.size()) - 1;
    d.n_bwd_lev = static_cast<int32_t>(p.bwd_lev_ptr.size()) - 1;
    d.n_tbw_lev = static_cast<int32_t>(p.tbw_lev_ptr.size()) - 1;
    d.max_col = p.max_col;
    d.nnz_l = p.lrow_ptr[p.n];
    d.nnz_u = p.urow_ptr[p.n];
    d.kind = p.kind;
    d.has_map = p.has_update_map ? 1 : 0;
    d.map16 = p.map16() ? 1 : 0;
    // grow geometrically once for this plan, so a multi-gigabyte update map
    // is copied once (appending to an unreserved pool re-copies it)
    const size_t need = pool.size() + static_cast<size_t>(p.device_words()) + 4 * nsg::PA_COUNT + 4;
    if (pool.capacity() < need) pool.reserve(std::max(need, 2 * pool.capacity()));
    p.append_to(pool, d.off);
    d.words = p.device_words();
    // the span [off[0], off[0] + words) may run past the last array by the
    // alignment slack: keep it inside the pool
    pool.insert(pool.end(), 4 * nsg::PA_COUNT, 0);
    return d;
}


std::unique_ptr<nsg_topology> clone_topology(const nsg_topology& t) {
    if (!t.engine && !t.amd) throw std::logic_error("clone_topology: topology has no ordering engine");
    auto c = std::make_unique<nsg_topology>();
    if (t.engine) c->engine = std::make_unique<nsg::MarkowitzOrder>(*t.engine);
    if (t.amd) c->amd = std::make_unique<nsg::AmdLuFactor>(*t.amd);
    c->slot_elem = t.slot_elem;
    c->auto_fallback = t.auto_fallback;
    c->committed = t.committed;
    c->plan = t.plan;
    return c;
}

bool same_plan(const nsg::TopologyPlan& a, const nsg::TopologyPlan& b) {
    return a.kind == b.kind && a.n == b.n && a.perm_row == b.perm_row &&
           a.perm_col == b.perm_col && a.col_ptr == b.col_ptr && a.row_idx == b.row_idx &&
           a.lu_src == b.lu_src && a.piv_rank == b.piv_rank && a.gmin_pos == b.gmin_pos;
}

int intern_topology(std::vector<std::unique_ptr<nsg_topology>>& topos,
                    std::unique_ptr<nsg_topology> t) {
    for (size_t k = 0; k < topos.size(); ++k)
        if (same_plan(topos[k]->plan, t->plan)) return static_cast<int>(k);
    topos.push_back(std::move(t));
    return static_cast<int>(topos.size()) - 1;
}

int reorder_instance(std::vector<std::unique_ptr<nsg_topology>>& topos, int topo,
                     const double* values, double diag_gmin, int* new_topo) {
    auto c = clone_topology(*topos[topo]);
    const int rc = numeric_on_engine(*c, values, diag_gmin);
    if (rc != NSG_OK) return rc;
    rebuild_plan(*c);
    *new_topo = intern_topology(topos, std::move(c));
    return NSG_OK;
}

// First column of the grid-wide refactor's CTA-mode tail for an AMD-LU plan:
// the longest suffix of columns that each apply at least kGridTailUpdates
// updates (the top separators, whose updates would otherwise run serially
// in one warp each); n (no tail) for Markowitz plans or a suffix shorter
// than two columns.
int32_t grid_tail_from(const nsg::TopologyPlan& p) {
    constexpr int32_t kGridTailUpdates = 128;
    if (p.kind != nsg::kPlanKindAmdLu || p.n < 2) return p.n;
    int32_t j = p.n;
    while (j > 0 && p.diag_pos[j - 1] - p.col_ptr[j - 1] >= kGridTailUpdates) --j;
    return (p.n - j >= 2) ? j : p.n;
}

void place_lu_workspace(nsg::DcDesc& d, const nsg::TopologyPlan& p, int64_t& work_size) {
    auto take = [&](int64_t n) {
        const int64_t off = work_size;
        work_size += (n + 3) & ~int64_t{3};
        return off;
    };
    d.lu_off = take(p.nnz_lu);
    d.lrows_off = take(p.lrow_ptr[p.n]);
    d.urows_off = take(p.urow_ptr[p.n]);
}

cudaError_t grow_workspace(double** d_work, int64_t* capacity, int64_t needed) {
    if (needed <= *capacity) return cudaSuccess;
    const int64_t cap = needed + needed / 4;
    double* w = nullptr;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&w), sizeof(double) * cap);
    if (e != cudaSuccess) return e;
    e = cudaMemcpy(w, *d_work, sizeof(double) * (*capacity), cudaMemcpyDeviceToDevice);
    if (e != cudaSuccess) {
        cudaFree(w);
        return e;
    }
    cudaFree(*d_work);
    *d_work = w;
    *capacity = cap;
    return cudaSuccess;
}

int refresh_plans(const std::vector<std::unique_ptr<nsg_topology>>& topos, int32_t** d_lu_pool,
                  nsg::PlanDesc** d_plans, int* max_col, int* max_n) {
    std::vector<int32_t> pool;
    std::vector<nsg::PlanDesc> plans;
    for (const auto& t : topos) {
        if (!t->plan.has_update_map)
            return fail(NSG_ERR_INVALID, "circuit too large for the batched Newton kernels");
        plans.push_back(make_plan_desc(t->plan, pool));
        *max_col = std::max(*max_col, t->plan.max_col);
        *max_n = std::max(*max_n, t->plan.n);
    }
    int32_t* p = nullptr;
    nsg::PlanDesc* q = nullptr;
    cudaError_t e;
    if ((e = upload(&p, pool.data(), pool.size())) != cudaSuccess ||
        (e = upload(&q, plans.data(), plans.size())) != cudaSuccess) {
        cudaFree(p);
        cudaFree(q);
        return cuda_fail("refresh_plans", e);
    }
    cudaFree(*d_lu_pool);
    cudaFree(*d_plans);
    *d_lu_pool = p;
    *d_plans = q;
    return NSG_OK;
}

}  // namespace nsg_internal

using namespace nsg_internal;

extern "C" {

const char* nsg_last_error(void) { return nsg_internal::g_last_error.c_str(); }

int nsg_set_wait_limit(int polls) {
    if (polls < 0) return fail(NSG_ERR_INVALID, "nsg_set_wait_limit: negative poll count");
    for (auto set : nsg::wait_limit_setters()) {
        const cudaError_t e = set(polls);
        if (e != cudaSuccess) return cuda_fail("nsg_set_wait_limit", e);
    }
    return NSG_OK;
}

int nsg_topology_order(int n, int nnz, const int* col_ptr, const int* row_idx,
                       const double* values, double diag_gmin, nsg_topology** out) {
    return guarded("nsg_topology_order", [&]() -> int {
        if (!out) return fail(NSG_ERR_INVALID, "nsg_topology_order: null out");
        *out = nullptr;
        std::unique_ptr<nsg_topology> t;
        const int rc = order_topology(n, nnz, col_ptr, row_idx, values, diag_gmin, t);
        if (rc == NSG_OK) *out = t.release();
        return rc;
    });
}

int nsg_topology_order_solver(int n, int nnz, const int* col_ptr, const int* row_idx,
                              const double* values, double diag_gmin, int solver,
                              nsg_topology** out) {
    return guarded("nsg_topology_order_solver", [&]() -> int {
        if (!out) return fail(NSG_ERR_INVALID, "nsg_topology_order_solver: null out");
        *out = nullptr;
        std::unique_ptr<nsg_topology> t;
        const int rc = order_topology(n, nnz, col_ptr, row_idx, values, diag_gmin, t, solver);
        if (rc == NSG_OK) *out = t.release();
        return rc;
    });
}

int nsg_solver_select(int num_vars, int is_linear) {
    return select_solver(num_vars, is_linear != 0);
}

int nsg_topology_solver(const nsg_topology* topo) {
    if (!topo) return fail(NSG_ERR_INVALID, "nsg_topology_solver: null topology");
    return topo->plan.kind == nsg::kPlanKindAmdLu ? NSG_SOLVER_AMDLU : NSG_SOLVER_MARKOWITZ;
}

int nsg_amd_order(int n, const int* col_ptr, const int* row_idx, int* perm) {
    return guarded("nsg_amd_order", [&]() -> int {
        if (n <= 0 || !col_ptr || !row_idx || !perm)
            return fail(NSG_ERR_INVALID, "nsg_amd_order: bad arguments");
        if (col_ptr[0] != 0 || !valid_csc(n, col_ptr, row_idx))
            return fail(NSG_ERR_INVALID, "nsg_amd_order: malformed pattern");
        const std::vector<int32_t> q = nsg::amd_order(n, col_ptr, row_idx);
        std::memcpy(perm, q.data(), sizeof(int) * q.size());
        return NSG_OK;
    });
}

int nsg_topology_numeric(nsg_topology* topo, const double* values, double diag_gmin,
                         int* reordered) {
    return guarded("nsg_topology_numeric", [&]() -> int {
        if (!topo || !values) return fail(NSG_ERR_INVALID, "nsg_topology_numeric: bad arguments");
        if (!topo->engine && !topo->amd)
            return fail(NSG_ERR_INVALID,
                        "nsg_topology_numeric: imported topology has no ordering state");
        if (topo->amd) {
            // AmdLuSolver::numeric: a full factor_ with fresh pivots.
            const int rc = numeric_on_engine(*topo, values, diag_gmin);
            if (rc != NSG_OK) {
                if (reordered) *reordered = 0;
                return fail(rc, "nsg_topology_numeric: singular matrix");
            }
            nsg_topology probe;
            probe.plan = topo->plan;
            rebuild_plan(*topo);
            if (reordered) *reordered = same_plan(probe.plan, topo->plan) ? 0 : 1;
            return NSG_OK;
        }
        const int before = topo->engine->fillin_count();
        const int rc = numeric_on_engine(*topo, values, diag_gmin);
        const int step = topo->engine->reorder_step();
        if (reordered) *reordered = step;
        if (rc != NSG_OK) return fail(rc, "nsg_topology_numeric: singular matrix");
        if (step != 0 || topo->engine->fillin_count() != before) rebuild_plan(*topo);
        return NSG_OK;
    });
}

int nsg_topology_import(int n, int nnz, const int* int_to_ext_row, const int* int_to_ext_col,
                        int n_elem, const int* elem_row, const int* elem_col,
                        const int* slot_to_elem, nsg_topology** out) {
    return guarded("nsg_topology_import", [&]() -> int {
        if (!out || !int_to_ext_row || !int_to_ext_col || !elem_row || !elem_col || !slot_to_elem)
            return fail(NSG_ERR_INVALID, "nsg_topology_import: null argument");
        *out = nullptr;
        auto t = std::make_unique<nsg_topology>();
        t->plan = nsg::build_plan_from_structure(n, nnz, int_to_ext_row, int_to_ext_col, n_elem,
                                                 elem_row, elem_col, slot_to_elem);
        *out = t.release();
        return NSG_OK;
    });
}

int nsg_topology_info(const nsg_topology* topo, int* n, int* nnz, int* nnz_lu,
                      long long* updates, int* col_levels, int* fwd_levels, int* bwd_levels) {
    if (!topo) return fail(NSG_ERR_INVALID, "nsg_topology_info: null topology");
    const auto& p = topo->plan;
    if (n) *n = p.n;
    if (nnz) *nnz = p.nnz_a;
    if (nnz_lu) *nnz_lu = p.nnz_lu;
    if (updates) *updates = p.updates;
    if (col_levels) *col_levels = static_cast<int>(p.col_lev_ptr.size()) - 1;
    if (fwd_levels) *fwd_levels = static_cast<int>(p.fwd_lev_ptr.size()) - 1;
    if (bwd_levels) *bwd_levels = static_cast<int>(p.bwd_lev_ptr.size()) - 1;
    return NSG_OK;
}

int nsg_topology_export(const nsg_topology* topo, int* int_to_ext_row, int* int_to_ext_col,
                        int* elem_row, int* elem_col, int* slot_to_elem) {
    if (!topo) return fail(NSG_ERR_INVALID, "nsg_topology_export: null topology");
    const auto& p = topo->plan;
    for (int i = 0; i < p.n; ++i) {
        if (int_to_ext_row) int_to_ext_row[i] = p.perm_row[i] + 1;
        if (int_to_ext_col) int_to_ext_col[i] = p.perm_col[i] + 1;
    }
    for (int j = 0; j < p.n; ++j)
        for (int q = p.col_ptr[j]; q < p.col_ptr[j + 1]; ++q) {
            if (elem_row) elem_row[q] = p.row_idx[q] + 1;
            if (elem_col) elem_col[q] = j + 1;
        }
    if (slot_to_elem) std::memcpy(slot_to_elem, p.a_to_lu.data(), sizeof(int) * p.nnz_a);
    return NSG_OK;
}

int nsg_topology_order_complex(int n, int nnz, const int* col_ptr, const int* row_idx,
                               const double* ax, nsg_topology** out) {
    return guarded("nsg_topology_order_complex", [&]() -> int {
        if (!out || n <= 0 || nnz <= 0 || !col_ptr || !row_idx || !ax)
            return fail(NSG_ERR_INVALID, "nsg_topology_order_complex: bad arguments");
        *out = nullptr;
        if (col_ptr[0] != 0 || col_ptr[n] != nnz || !valid_csc(n, col_ptr, row_idx))
            return fail(NSG_ERR_INVALID, "nsg_topology_order_complex: malformed CSC pattern");
        auto t = std::make_unique<nsg_topology>();
        make_markowitz(*t, n, col_ptr, row_idx);
        t->committed = true;
        auto& mo = *t->engine;
        // NeoSolver::numeric_complex (src/core/neo_solver.cpp:228-245):
        // load_complex, the MNA pre-order, order_and_factor(relThr 1e-3,
        // absThr 1e-13, diagonal pivoting) on the complex values.
        mo.set_complex(true);
        mo.clear_fillins();
        for (size_t k = 0; k < t->slot_elem.size(); ++k) {
            mo.value(t->slot_elem[k]) = ax[2 * k];
            mo.value_imag(t->slot_elem[k]) = ax[2 * k + 1];
        }
        mo.mna_preorder();
        const nsg::OrderStatus st = mo.order_and_factor(1e-3, 1e-13, true);
        if (st == nsg::OrderStatus::no_memory)
            return fail(NSG_ERR_NOMEM, "nsg_topology_order_complex: out of memory");
        if (st == nsg::OrderStatus::singular)
            return fail(NSG_SINGULAR, "nsg_topology_order_complex: singular matrix");
        rebuild_plan(*t);
        *out = t.release();
        return NSG_OK;
    });
}

void nsg_topology_free(nsg_topology* topo) { delete topo; }

int nsg_batch_create(int count, nsg_topology* const* topos, nsg_batch** out) {
    return guarded("nsg_batch_create", [&]() -> int {
        if (!out || count <= 0 || !topos)
            return fail(NSG_ERR_INVALID, "nsg_batch_create: bad arguments");
        *out = nullptr;
        auto b = std::make_unique<nsg_batch>();
        b->count = count;
        cudaError_t de = cudaGetDevice(&b->device);
        if (de != cudaSuccess) return cuda_fail("nsg_batch_create: current device", de);
        std::unordered_map<const nsg_topology*, int32_t> plan_of;
        std::vector<nsg::PlanDesc> plans;
        std::vector<int32_t> pool;
        std::vector<nsg::InstDesc> insts(count);
        b->a_off.assign(count + 1, 0);
        b->x_off.assign(count + 1, 0);
        b->lu_off.assign(count + 1, 0);
        int64_t lrows = 0, urows = 0;
        for (int i = 0; i < count; ++i) {
            const nsg_topology* t = topos[i];
            if (!t) return fail(NSG_ERR_INVALID, "nsg_batch_create: null topology");
            auto it = plan_of.find(t);
            if (it == plan_of.end()) {
                it = plan_of.emplace(t, static_cast<int32_t>(plans.size())).first;
                plans.push_back(make_plan_desc(t->plan, pool));
            }
            const auto& p = t->plan;
            if (!p.has_update_map) b->unmapped = true;
            b->max_col = std::max(b->max_col, p.max_col);
            b->max_n = std::max(b->max_n, p.n);
            insts[i].plan = it->second;
            insts[i].index = i;
            insts[i].a_off = b->a_off[i];
            insts[i].lu_off = b->lu_off[i];
            insts[i].x_off = b->x_off[i];
            insts[i].w_off = b->x_off[i];
            insts[i].lrows_off = lrows;
            insts[i].urows_off = urows;
            lrows += (p.lrow_ptr[p.n] + 3) & ~3;
            urows += (p.urow_ptr[p.n] + 3) & ~3;
            b->a_off[i + 1] = b->a_off[i] + p.nnz_a;
            b->x_off[i + 1] = b->x_off[i] + p.n;
            // keep each instance's LU 32-byte aligned
            b->lu_off[i + 1] = b->lu_off[i] + ((p.nnz_lu + 3) & ~3);
        }
        // Largest instances first: the grid's tail is made of small ones.
        std::stable_sort(insts.begin(), insts.end(), [&](const nsg::InstDesc& x, const nsg::InstDesc& y) {
            return topos[x.index]->plan.updates > topos[y.index]->plan.updates;
        });
        // Unknowns per launch slot (the grid-wide schedule walks insts[]).
        for (const auto& d : insts) {
            b->n_of.push_back(topos[d.index]->plan.n);
            b->tail_from_of.push_back(grid_tail_from(topos[d.index]->plan));
            b->amd_of.push_back(topos[d.index]->plan.kind == nsg::kPlanKindAmdLu ? 1 : 0);
        }
        cudaError_t e;
        if ((e = upload(&b->d_pool, pool.data(), pool.size())) != cudaSuccess ||
            (e = upload(&b->d_plans, plans.data(), plans.size())) != cudaSuccess ||
            (e = upload(&b->d_insts, insts.data(), insts.size())) != cudaSuccess ||
            (e = upload<double>(&b->d_lu, nullptr, b->lu_off[count])) != cudaSuccess ||
            (e = upload<double>(&b->d_work, nullptr, b->x_off[count])) != cudaSuccess ||
            (e = upload<double>(&b->d_lrows, nullptr, lrows)) != cudaSuccess ||
            (e = upload<double>(&b->d_urows, nullptr, urows)) != cudaSuccess)
            return cuda_fail("nsg_batch_create", e);
        // A plan too large for an update map runs only on the grid-wide
        // schedule (per-warp row maps instead).
        if (b->unmapped) {
            b->schedule = 2;
            b->allow_flow = false;
        }
        *out = b.release();
        return NSG_OK;
    });
}

void nsg_batch_free(nsg_batch* batch) { delete batch; }

int nsg_batch_refactor_complex(nsg_batch* b, const double* d_ax, double* d_lu, int* d_status,
                               void* stream) {
    if (!b || !d_ax || !d_lu || !d_status)
        return fail(NSG_ERR_INVALID, "nsg_batch_refactor_complex: null argument");
    if (b->unmapped)
        return fail(NSG_ERR_INVALID, "nsg_batch_refactor_complex: topology too large for an "
                                     "update map");
    const size_t smem = nsg::complex_refactor_smem(b->max_n);
    if (smem > 200 * 1024)
        return fail(NSG_ERR_INVALID, "nsg_batch_refactor_complex: too many unknowns per instance "
                                     "for the shared-memory completion flags");
    const cudaError_t e = nsg::launch_complex_refactor(b->d_plans, b->d_pool, b->d_insts, b->count,
                                                       b->max_n, d_ax, d_lu, d_status,
                                                       static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? NSG_OK : cuda_fail("nsg_batch_refactor_complex", e);
}

int nsg_batch_solve_complex(nsg_batch* b, const double* d_lu, double* d_x, void* stream) {
    if (!b || !d_lu || !d_x) return fail(NSG_ERR_INVALID, "nsg_batch_solve_complex: null argument");
    cudaError_t e = cudaSuccess;
    if (!b->d_cwork) {
        e = cudaMalloc(reinterpret_cast<void**>(&b->d_cwork),
                       sizeof(double) * 2 * static_cast<size_t>(std::max<long long>(1, b->x_off[b->count])));
        if (e != cudaSuccess) return cuda_fail("nsg_batch_solve_complex: workspace", e);
    }
    e = nsg::launch_complex_solve(b->d_plans, b->d_pool, b->d_insts, b->count, d_lu, d_x,
                                  b->d_cwork, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? NSG_OK : cuda_fail("nsg_batch_solve_complex", e);
}

int nsg_batch_layout(const nsg_batch* b, long long* value_offsets, long long* vector_offsets,
                     long long* lu_offsets) {
    if (!b) return fail(NSG_ERR_INVALID, "nsg_batch_layout: null batch");
    const size_t bytes = sizeof(long long) * (b->count + 1);
    if (value_offsets) std::memcpy(value_offsets, b->a_off.data(), bytes);
    if (vector_offsets) std::memcpy(vector_offsets, b->x_off.data(), bytes);
    if (lu_offsets) std::memcpy(lu_offsets, b->lu_off.data(), bytes);
    return NSG_OK;
}

int nsg_batch_refactor(nsg_batch* b, const double* d_values, double diag_gmin,
                       int check_pivots, int* d_status, int* d_fail_step, void* stream) {
    if (!b || !d_values || !d_status)
        return fail(NSG_ERR_INVALID, "nsg_batch_refactor: null argument");
    // check_pivots: a numeric() (re-validate / re-choose the pivots), else a
    // refactorize() (AMD-LU topologies run the replay's growth test).
    const int mode = check_pivots ? nsg::kCheckNumeric : nsg::kCheckRefactor;
    if (b->schedule == 2) {
        if (!b->d_grid) {
            cudaError_t e = cudaMalloc(&b->d_grid, nsg::grid_scratch_bytes(b->max_n));
            if (e != cudaSuccess) return cuda_fail("nsg_batch_refactor", e);
        }
        if (b->unmapped) {
            const int64_t words = nsg::grid_rmap_words(b->grid_colbuf, b->max_col, b->max_n);
            if (words > b->rmap_cap) {
                cudaFree(b->d_rmap);
                b->d_rmap = nullptr;
                b->rmap_cap = 0;
                cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&b->d_rmap),
                                           sizeof(int32_t) * static_cast<size_t>(words));
                if (e != cudaSuccess) return cuda_fail("nsg_batch_refactor", e);
                b->rmap_cap = words;
            }
        }
        std::vector<int32_t> cta_from(b->n_of);
        for (int i = 0; i < b->count; ++i) {
            if (b->grid_tail < 0) cta_from[i] = b->tail_from_of[i];
            else if (b->amd_of[i]) cta_from[i] = std::max(0, b->n_of[i] - b->grid_tail);
        }
        cudaError_t e = nsg::launch_grid_refactor(
            b->d_plans, b->d_pool, b->d_insts, b->count, b->n_of.data(), d_values, b->d_lu,
            diag_gmin, mode, 1e-3, d_status, d_fail_step, b->d_lrows, b->d_urows, b->d_grid,
            b->grid_colbuf, b->max_col, b->unmapped ? b->d_rmap : nullptr, b->max_n,
            cta_from.data(), static_cast<cudaStream_t>(stream));
        if (e == cudaSuccess) b->rows_valid = true;
        return e == cudaSuccess ? NSG_OK : cuda_fail("nsg_batch_refactor", e);
    }
    cudaError_t e = nsg::launch_refactor(b->d_plans, b->d_pool, b->d_insts, b->count, d_values,
                                         b->d_lu, diag_gmin, mode, 1e-3, d_status,
                                         d_fail_step, b->max_col, b->max_n, b->allow_flow,
                                         b->d_lrows, b->d_urows, static_cast<cudaStream_t>(stream));
    if (e == cudaSuccess) b->rows_valid = b->allow_flow;
    return e == cudaSuccess ? NSG_OK : cuda_fail("nsg_batch_refactor", e);
}

int nsg_batch_solve(nsg_batch* b, double* d_x, void* stream) {
    if (!b || !d_x) return fail(NSG_ERR_INVALID, "nsg_batch_solve: null argument");
    if (b->schedule == 2 && b->rows_valid && b->d_grid) {
        cudaError_t e = nsg::launch_grid_solve(b->d_plans, b->d_pool, b->d_insts, b->count,
                                               b->n_of.data(), b->d_lu, b->d_lrows, b->d_urows,
                                               d_x, b->d_work, b->d_grid,
                                               static_cast<cudaStream_t>(stream));
        return e == cudaSuccess ? NSG_OK : cuda_fail("nsg_batch_solve", e);
    }
    cudaError_t e = nsg::launch_solve(b->d_plans, b->d_pool, b->d_insts, b->count, b->d_lu, d_x,
                                      b->d_work, false, b->rows_valid ? b->d_lrows : nullptr,
                                      b->d_urows, b->max_n, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? NSG_OK : cuda_fail("nsg_batch_solve", e);
}

int nsg_batch_solve_transposed(nsg_batch* b, double* d_x, void* stream) {
    if (!b || !d_x) return fail(NSG_ERR_INVALID, "nsg_batch_solve_transposed: null argument");
    cudaError_t e = nsg::launch_solve(b->d_plans, b->d_pool, b->d_insts, b->count, b->d_lu, d_x,
                                      b->d_work, true, nullptr, nullptr, b->max_n,
                                      static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? NSG_OK : cuda_fail("nsg_batch_solve_transposed", e);
}

const double* nsg_batch_lu(const nsg_batch* b) { return b ? b->d_lu : nullptr; }

int nsg_set_update_map_limit(long long words) {
    if (words < 0) return fail(NSG_ERR_INVALID, "nsg_set_update_map_limit: negative limit");
    nsg::set_update_map_limit(words);
    return NSG_OK;
}

int nsg_batch_set_grid_tail(nsg_batch* b, int columns) {
    if (!b || columns < -1) return fail(NSG_ERR_INVALID, "nsg_batch_set_grid_tail: bad arguments");
    b->grid_tail = columns;
    return NSG_OK;
}

int nsg_batch_set_grid_buffer(nsg_batch* b, int doubles) {
    if (!b || (doubles != 0 && doubles != 1024 && doubles != 2048 && doubles != 4096))
        return fail(NSG_ERR_INVALID, "nsg_batch_set_grid_buffer: bad arguments");
    b->grid_colbuf = doubles;
    return NSG_OK;
}

int nsg_batch_set_schedule(nsg_batch* b, int schedule) {
    if (!b || schedule < 0 || schedule > 2)
        return fail(NSG_ERR_INVALID, "nsg_batch_set_schedule: bad arguments");
    if (b->unmapped && schedule != 2)
        return fail(NSG_ERR_INVALID, "nsg_batch_set_schedule: a topology of this batch is too "
                                     "large for an update map; only schedule 2 runs it");
    b->allow_flow = (schedule == 0);
    b->schedule = schedule;
    b->rows_valid = false;
    return NSG_OK;
}

int nsg_batch_autotune(nsg_batch* b, const double* d_values, double* d_x, int reps,
                       float* times_ms, int* chosen, void* stream) {
    return guarded("nsg_batch_autotune", [&]() -> int {
        if (!b || !d_values || !d_x || reps < 1)
            return fail(NSG_ERR_INVALID, "nsg_batch_autotune: bad arguments");
        const cudaStream_t st = static_cast<cudaStream_t>(stream);
        const size_t nx = static_cast<size_t>(b->x_off[b->count]);
        double* d_b = nullptr;
        int32_t* d_st = nullptr;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&d_b), sizeof(double) * nx);
        if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&d_st), sizeof(int32_t) * b->count);
        if (e == cudaSuccess) e = cudaEventCreate(&e0);
        if (e == cudaSuccess) e = cudaEventCreate(&e1);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_b, d_x, sizeof(double) * nx, cudaMemcpyDeviceToDevice, st);
        const int saved = b->schedule;
        int best = -1;
        float best_ms = 0.0f;
        // Refactor (a refactorize(), as the Newton loop's steady state) and
        // solve of the given system under each schedule, reps times.
        for (int sched = 0; sched < 3 && e == cudaSuccess; ++sched) {
            float ms = -1.0f;
            int rc = nsg_batch_set_schedule(b, sched);
            auto once = [&]() -> int {
                int r = nsg_batch_refactor(b, d_values, 0.0, 0, d_st, nullptr, stream);
                if (r == NSG_OK &&
                    (e = cudaMemcpyAsync(d_x, d_b, sizeof(double) * nx, cudaMemcpyDeviceToDevice,
                                         st)) != cudaSuccess)
                    return NSG_ERR_CUDA;
                if (r == NSG_OK) r = nsg_batch_solve(b, d_x, stream);
                return r;
            };
            if (rc == NSG_OK) rc = once();  // warm-up (allocates scratch)
            if (rc == NSG_OK && (e = cudaEventRecord(e0, st)) == cudaSuccess) {
                for (int k = 0; k < reps && rc == NSG_OK; ++k) rc = once();
                if (rc == NSG_OK && (e = cudaEventRecord(e1, st)) == cudaSuccess &&
                    (e = cudaEventSynchronize(e1)) == cudaSuccess &&
                    (e = cudaEventElapsedTime(&ms, e0, e1)) == cudaSuccess)
                    ms /= static_cast<float>(reps);
            }
            if (rc != NSG_OK || e != cudaSuccess) ms = -1.0f;
            if (times_ms) times_ms[sched] = ms;
            if (ms >= 0.0f && (best < 0 || ms < best_ms)) {
                best = sched;
                best_ms = ms;
            }
        }
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_x, d_b, sizeof(double) * nx, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaFree(d_b);
        cudaFree(d_st);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (e != cudaSuccess) return cuda_fail("nsg_batch_autotune", e);
        if (best < 0) {
            nsg_batch_set_schedule(b, saved);
            return fail(NSG_ERR_INVALID, "nsg_batch_autotune: no schedule ran");
        }
        nsg_batch_set_schedule(b, best);
        if (chosen) *chosen = best;
        return NSG_OK;
    });
}

int nsg_batch_lu_to_host(const nsg_batch* b, double* out) {
    if (!b || !out) return fail(NSG_ERR_INVALID, "nsg_batch_lu_to_host: null argument");
    cudaError_t e = cudaMemcpy(out, b->d_lu, sizeof(double) * b->lu_off[b->count],
                               cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? NSG_OK : cuda_fail("nsg_batch_lu_to_host", e);
}

}  // extern "C"
