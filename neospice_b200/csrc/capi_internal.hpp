// Internal definitions shared by the C ABI translation units.
#pragma once
#include "nsgpu.h"

#include "host/amd_lu.hpp"
#include "host/circuit.hpp"
#include "host/plan.hpp"
#include "host/sparse_order.hpp"
#include "kernels/dc_device.cuh"
#include "kernels/lu_device.cuh"

#include <cuda_runtime.h>

#include <exception>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

// One symbolic result.  Exactly one engine is set for a topology that can
// re-order: the Markowitz engine (NeoSolver) or the AMD-LU engine
// (AmdLuSolver); an imported topology has neither.
struct nsg_topology {
    std::unique_ptr<nsg::MarkowitzOrder> engine;
    std::vector<int32_t> slot_elem;  // Markowitz: engine element of each caller slot
    std::unique_ptr<nsg::AmdLuFactor> amd;
    // make_solver's AutoFallbackSolver (make_solver.cpp:71-145): an AMD-LU
    // engine that switches to Markowitz for good when its first
    // factorization is singular.
    bool auto_fallback = false;
    bool committed = false;  // a first factorization has been attempted
    nsg::TopologyPlan plan;
};

struct nsg_circuit {
    explicit nsg_circuit(int nodes) : c(nodes) {}
    nsg::Circuit c;
};

struct nsg_batch {
    int count = 0;
    int device = 0;  // the CUDA device current when the batch was created
    std::vector<long long> a_off, x_off, lu_off;
    int32_t* d_pool = nullptr;
    nsg::PlanDesc* d_plans = nullptr;
    nsg::InstDesc* d_insts = nullptr;
    double* d_lu = nullptr;
    double* d_work = nullptr;
    double* d_lrows = nullptr;  // row-major L copy written by the dataflow refactor
    double* d_urows = nullptr;  // row-major U copy
    bool rows_valid = false;    // the copies match d_lu (last refactor was dataflow)
    int max_col = 0;
    int max_n = 0;
    bool allow_flow = true;
    int schedule = 0;             // nsg_batch_set_schedule
    int grid_colbuf = 0;          // nsg_batch_set_grid_buffer (0: automatic)
    bool unmapped = false;        // a plan has no update map (grid-wide schedule only)
    int32_t* d_rmap = nullptr;    // per-warp row -> position maps of such plans
    int64_t rmap_cap = 0;         // words allocated at d_rmap
    std::vector<int32_t> n_of;    // unknowns of the instance in each slot of d_insts
    // Grid-wide refactor: per slot, the first column claimed by whole CTAs
    // (the chosen tail; n for none), and nsg_batch_set_grid_tail's setting
    // (-1: the tail of columns with at least kGridTailUpdates U entries).
    std::vector<int32_t> tail_from_of;
    std::vector<char> amd_of;     // the slot's plan is AMD-LU (CTA mode needs it)
    int grid_tail = -1;
    void* d_grid = nullptr;       // flags and state of the grid-wide schedule
    double* d_cwork = nullptr;    // complex sweep workspace (2 doubles per unknown)
    ~nsg_batch() {
        cudaFree(d_rmap);
        cudaFree(d_cwork);
        cudaFree(d_grid);
        cudaFree(d_pool);
        cudaFree(d_plans);
        cudaFree(d_insts);
        cudaFree(d_lu);
        cudaFree(d_work);
        cudaFree(d_lrows);
        cudaFree(d_urows);
    }
};

namespace nsg_internal {

int fail(int code, const std::string& msg);
int cuda_fail(const char* where, cudaError_t e);
void clear_error();

// Run a body, mapping C++ exceptions to status codes.
template <class F>
int guarded(const char* where, F&& body) {
    try {
        clear_error();
        return body();
    } catch (const std::bad_alloc&) {
        return fail(NSG_ERR_NOMEM, std::string(where) + ": out of host memory");
    } catch (const std::exception& e) {
        return fail(NSG_ERR_INVALID, std::string(where) + ": " + e.what());
    }
}

template <class T>
cudaError_t upload(T** dst, const T* src, size_t count) {
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(dst), count * sizeof(T));
    if (e != cudaSuccess) return e;
    if (src) e = cudaMemcpy(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice);
    return e;
}

// numeric() of the topology's engine on the host: NeoSolver's load,
// preorder, gmin and ordering, or AmdLuSolver's full factor_ (with the
// AutoFallbackSolver switch on a singular first factorization).
int numeric_on_engine(nsg_topology& t, const double* values, double diag_gmin);
// Rebuild t.plan from its engine after a successful numeric_on_engine.
void rebuild_plan(nsg_topology& t);

// make_solver's choice (make_solver.cpp:156-178) for a circuit: NSG_SOLVER_*.
int select_solver(int num_vars, bool is_linear);

// nsg_topology_order without the C wrapper (throws on bad input); solver is
// an NSG_SOLVER_* engine.
int order_topology(int n, int nnz, const int* col_ptr, const int* row_idx, const double* values,
                   double diag_gmin, std::unique_ptr<nsg_topology>& out,
                   int solver = NSG_SOLVER_MARKOWITZ);

// PlanDesc for a plan whose arrays were appended to pool.
nsg::PlanDesc make_plan_desc(const nsg::TopologyPlan& p, std::vector<int32_t>& pool);

}  // namespace nsg_internal

namespace nsg { struct DcDesc; }
namespace nsg_internal {
void fill_instance(nsg::DcDesc& d, const nsg::Circuit& c, const nsg::TopologyPlan& p,
                   std::vector<int32_t>& prog, int64_t& work);
// The gmin-stepping save area, placed after the staged regions.
void place_dcsave(nsg::DcDesc& d, int64_t& work);
// Largest stage_len over instances (doubles).
inline int64_t max_stage_len(const std::vector<nsg::DcDesc>& ds) {
    int64_t m = 0;
    for (const auto& d : ds) m = d.stage_len > m ? d.stage_len : m;
    return m;
}

// Host (re-)ordering of one instance that stopped on the device.
// reorder_instance: a copy of topos[topo]'s engine runs NeoSolver::numeric on
// the instance's matrix values (re-validate, re-order from the failing
// step); the result is shared with an existing topology of identical
// structure (intern_topology) or appended.  *new_topo receives its index.
std::unique_ptr<nsg_topology> clone_topology(const nsg_topology& t);
bool same_plan(const nsg::TopologyPlan& a, const nsg::TopologyPlan& b);
int intern_topology(std::vector<std::unique_ptr<nsg_topology>>& topos,
                    std::unique_ptr<nsg_topology> t);
int reorder_instance(std::vector<std::unique_ptr<nsg_topology>>& topos, int topo,
                     const double* values, double diag_gmin, int* new_topo);
// Fresh LU / row-copy regions for a re-ordered instance at the end of the
// workspace (work_size grows).
int32_t grid_tail_from(const nsg::TopologyPlan& p);
void place_lu_workspace(nsg::DcDesc& d, const nsg::TopologyPlan& p, int64_t& work_size);
// Reallocate the device workspace to hold `needed` doubles, keeping contents.
cudaError_t grow_workspace(double** d_work, int64_t* capacity, int64_t needed);
// Rebuild and re-upload the plan pool and descriptors of all topologies.
int refresh_plans(const std::vector<std::unique_ptr<nsg_topology>>& topos, int32_t** d_lu_pool,
                  nsg::PlanDesc** d_plans, int* max_col, int* max_n);
}  // namespace nsg_internal
