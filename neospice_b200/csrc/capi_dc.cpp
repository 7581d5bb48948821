// C ABI of circuits and batched DC operating points (include/nsgpu.h).
#include "capi_internal.hpp"

#include "host/circuit.hpp"
#include "kernels/mos1_model.cuh"
#include "kernels/dc_device.cuh"

#include <algorithm>
#include <cmath>
#include <atomic>
#include <cstring>
#include <map>
#include <thread>
#include <tuple>

namespace nsg {
cudaError_t launch_newton_dc(const PlanDesc* plans, const int32_t* lu_pool, const DcDesc* descs,
                             const int32_t* subset, int count, const int32_t* prog,
                             const double* params, double* work, double* solutions,
                             int32_t* status, int32_t* iterations, DcCtl* ctls,
                             const NewtonOptions& opt, int max_col, int max_n,
                             long long max_stage, int32_t* rmaps, cudaStream_t stream);
size_t dc_smem_bytes(int max_col, int max_n);
cudaError_t launch_dc_adjoint(const PlanDesc* plans, const int32_t* lu_pool, const DcDesc* descs,
                              int count, const int32_t* prog, const double* params, double* work,
                              const double* solutions, const double* cotangent, double* grads,
                              int32_t* status, const NewtonOptions& opt, int max_col, int max_n,
                              cudaStream_t stream);
}  // namespace nsg

using namespace nsg_internal;

struct nsg_dc_batch {
    int count = 0;
    std::vector<std::unique_ptr<nsg_topology>> topos;  // distinct symbolic results
    std::vector<long long> param_off, sol_off;
    std::vector<long long> inst_n, inst_nnz, inst_nnz_lu, inst_updates;
    std::vector<double> host_params;
    long long updates = 0, nnz_lu = 0, nnz = 0, n = 0;
    int max_col = 0, max_n = 0;
    nsg::NewtonOptions opt{1e-3, 1e-6, 1e-12, 1e-12, 0.0, 100, nsg::kAidDirect};
    bool row_maps = false;        // nsg_dc_batch_set_row_maps
    int32_t* d_rmap = nullptr;    // per-warp row -> position maps (count x warps x max_n)
    int64_t rmap_cap = 0;
    int32_t* d_lu_pool = nullptr;
    nsg::PlanDesc* d_plans = nullptr;
    int32_t* d_prog = nullptr;
    nsg::DcDesc* d_descs = nullptr;
    double* d_work = nullptr;
    double* d_params = nullptr;
    // Host re-ordering of instances whose pivots fail re-validation.
    bool reorder = true;
    long long reorders = 0;
    std::vector<nsg::DcDesc> descs;   // host copy, launch order
    std::vector<int> desc_pos;        // instance index -> position in descs
    std::vector<int> topo_of;         // instance index -> topology
    int64_t work_size = 0, work_cap = 0;
    nsg::DcCtl* d_ctl = nullptr;
    int32_t* d_subset = nullptr;
    // Graph replay of the launch (controller reset + Newton kernel), keyed
    // by the caller's buffers; dropped whenever plans or workspace move.
    bool use_graph = false;
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    const void* graph_key[4] = {nullptr, nullptr, nullptr, nullptr};
    long long graph_launches = 0, plain_launches = 0;
    void drop_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
    }
    ~nsg_dc_batch() {
        drop_graph();
        if (cap_stream) cudaStreamDestroy(cap_stream);
        cudaFree(d_rmap);
        cudaFree(d_lu_pool);
        cudaFree(d_plans);
        cudaFree(d_prog);
        cudaFree(d_descs);
        cudaFree(d_work);
        cudaFree(d_params);
        cudaFree(d_ctl);
        cudaFree(d_subset);
    }
};

namespace {

// Append an int vector to the pool at a 16-byte boundary; return its offset.
int64_t append(std::vector<int32_t>& pool, const std::vector<int32_t>& v) {
    while (pool.size() % 4) pool.push_back(0);
    const int64_t off = static_cast<int64_t>(pool.size());
    pool.insert(pool.end(), v.begin(), v.end());
    return off;
}

int64_t align4(int64_t x) { return (x + 3) & ~int64_t{3}; }

// Run f(i) for i in [0, count) on up to `threads` host threads.
template <class F>
void parallel_for(int count, int threads, F&& f) {
    threads = std::max(1, std::min(threads, count));
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    std::vector<std::exception_ptr> errs(threads);
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&, t] {
            try {
                for (int i; (i = next.fetch_add(1)) < count;) f(i);
            } catch (...) {
                errs[t] = std::current_exception();
            }
        });
    for (auto& th : pool) th.join();
    for (auto& e : errs)
        if (e) std::rethrow_exception(e);
}

}  // namespace

namespace nsg_internal {

// Program arrays and workspace of one instance (everything but index, plan,
// parameter and solution offsets).
void fill_instance(nsg::DcDesc& d, const nsg::Circuit& c, const nsg::TopologyPlan& p,
                   std::vector<int32_t>& prog, int64_t& work) {
    d.n = c.num_vars();
    d.num_nodes = c.num_nodes();
    d.nnz = c.nnz();
    d.n_const = c.n_const_terms();
    d.n_diodes = static_cast<int32_t>(c.diodes().size());
    d.n_caps = static_cast<int32_t>(c.caps().size());
    d.n_srcs = static_cast<int32_t>(c.wave_sources().size());
    d.n_mos = static_cast<int32_t>(c.mosfets().size());
    d.n_states = c.num_states();
    d.prog_off[nsg::DP_slot_ptr] = append(prog, c.slot_ptr());
    d.prog_off[nsg::DP_slot_terms] = append(prog, c.slot_terms());
    d.prog_off[nsg::DP_rhs_ptr] = append(prog, c.rhs_ptr());
    d.prog_off[nsg::DP_rhs_terms] = append(prog, c.rhs_terms());
    d.prog_off[nsg::DP_ucb_ptr] = append(prog, c.ucb_ptr());
    d.prog_off[nsg::DP_ucb_terms] = append(prog, c.ucb_terms());
    d.prog_off[nsg::DP_term_op] = append(prog, c.term_op());
    d.prog_off[nsg::DP_term_param] = append(prog, c.term_param());
    std::vector<int32_t> tab;
    for (const auto& dr : c.diodes()) tab.insert(tab.end(), {dr.pos, dr.neg, dr.param, dr.state});
    d.prog_off[nsg::DP_diodes] = append(prog, tab);
    tab.clear();
    for (const auto& cr : c.caps()) tab.insert(tab.end(), {cr.pos, cr.neg, cr.param, cr.has_ic, cr.state});
    d.prog_off[nsg::DP_caps] = append(prog, tab);
    tab.clear();
    for (const auto& sr : c.wave_sources()) tab.insert(tab.end(), {sr.is_voltage, sr.wave, sr.param, sr.nparam});
    d.prog_off[nsg::DP_srcs] = append(prog, tab);
    tab.clear();
    for (const auto& m : c.mosfets())
        tab.insert(tab.end(), {m.d, m.g, m.s, m.b, m.param, m.state, m.family});
    d.prog_off[nsg::DP_mos] = append(prog, tab);
    d.prog_off[nsg::DP_grad] = append(prog, c.grad_program());
    d.n_grad = static_cast<int32_t>(c.grad_program().size() / 5);
    d.x_off = work; work = align4(work + d.n);
    d.xold_off = work; work = align4(work + d.n);
    d.w_off = work; work = align4(work + d.n);
    d.a_off = work; work = align4(work + d.nnz);
    d.lu_off = work; work = align4(work + p.nnz_lu);
    d.lrows_off = work; work = align4(work + p.lrow_ptr[p.n]);
    d.urows_off = work; work = align4(work + p.urow_ptr[p.n]);
    d.tv_off = work; work = align4(work + c.n_terms());
    d.dconst_off = work; work = align4(work + 3 * d.n_diodes);
    d.state_off = work; work = align4(work + 4 * static_cast<int64_t>(d.n_states));
    d.mrec_off = work; work = align4(work + nsg::kMosRecCount * static_cast<int64_t>(d.n_mos));
    d.stage_len = work - d.x_off;
}

void place_dcsave(nsg::DcDesc& d, int64_t& work) {
    d.dcsave_off = work;
    work = align4(work + d.n + 3 * static_cast<int64_t>(d.n_states));
}

}  // namespace nsg_internal

extern "C" {

int nsg_circuit_create(int num_nodes, nsg_circuit** out) {
    return guarded("nsg_circuit_create", [&]() -> int {
        if (!out) return fail(NSG_ERR_INVALID, "nsg_circuit_create: null out");
        *out = new nsg_circuit(num_nodes);
        return NSG_OK;
    });
}

void nsg_circuit_free(nsg_circuit* c) { delete c; }

int nsg_circuit_add_resistor(nsg_circuit* c, int a, int b, double ohms) {
    return guarded("nsg_circuit_add_resistor", [&]() -> int {
        if (!c) return fail(NSG_ERR_INVALID, "null circuit");
        c->c.add_resistor(a, b, ohms);
        return NSG_OK;
    });
}

int nsg_circuit_add_vsource(nsg_circuit* c, int p, int n, double volts) {
    return guarded("nsg_circuit_add_vsource", [&]() -> int {
        if (!c) return fail(NSG_ERR_INVALID, "null circuit");
        c->c.add_vsource(p, n, volts);
        return NSG_OK;
    });
}

int nsg_circuit_add_isource(nsg_circuit* c, int p, int n, double amps) {
    return guarded("nsg_circuit_add_isource", [&]() -> int {
        if (!c) return fail(NSG_ERR_INVALID, "null circuit");
        c->c.add_isource(p, n, amps);
        return NSG_OK;
    });
}

int nsg_circuit_add_diode(nsg_circuit* c, int anode, int cathode, double is, double n_emission) {
    return guarded("nsg_circuit_add_diode", [&]() -> int {
        if (!c) return fail(NSG_ERR_INVALID, "null circuit");
        c->c.add_diode(anode, cathode, is, n_emission);
        return NSG_OK;
    });
}

int nsg_circuit_set_temperature(nsg_circuit* c, double kelvin) {
    return guarded("nsg_circuit_set_temperature", [&]() -> int {
        if (!c) return fail(NSG_ERR_INVALID, "null circuit");
        c->c.set_temperature(kelvin);
        return NSG_OK;
    });
}

int nsg_circuit_add_diode_card(nsg_circuit* c, int anode, int cathode, double is,
                               double n_emission, double cjo, double vj, double m, double fc,
                               double tt) {
    return guarded("nsg_circuit_add_diode_card", [&]() -> int {
        if (!c) return fail(NSG_ERR_INVALID, "null circuit");
        c->c.add_diode(anode, cathode, is, n_emission, cjo, vj, m, fc, tt);
        return NSG_OK;
    });
}

int nsg_circuit_add_diode_card_ex(nsg_circuit* c, int anode, int cathode, double is,
                                  double n_emission, double cjo, double vj, double m, double fc,
                                  double tt, double bv, double ibv, double nbv, double rs) {
    return guarded("nsg_circuit_add_diode_card_ex", [&]() -> int {
        if (!c) return fail(NSG_ERR_INVALID, "null circuit");
        c->c.add_diode(anode, cathode, is, n_emission, cjo, vj, m, fc, tt, bv, ibv, nbv, rs);
        return NSG_OK;
    });
}

int nsg_diode_param_block(double is, double n_emission, double cjo, double vj, double m,
                          double fc, double tt, double bv, double ibv, double nbv, double rs,
                          double* out) {
    return guarded("nsg_diode_param_block", [&]() -> int {
        if (!out) return fail(NSG_ERR_INVALID, "nsg_diode_param_block: null out");
        const std::vector<double> p =
            nsg::diode_param_block(is, n_emission, cjo, vj, m, fc, tt, bv, ibv, nbv, rs);
        std::copy(p.begin(), p.end(), out);
        return NSG_OK;
    });
}

int nsg_circuit_add_capacitor(nsg_circuit* c, int a, int b, double farads, int has_ic,
                              double ic) {
    return guarded("nsg_circuit_add_capacitor", [&]() -> int {
        if (!c) return fail(NSG_ERR_INVALID, "null circuit");
        c->c.add_capacitor(a, b, farads, has_ic != 0, ic);
        return NSG_OK;
    });
}

int nsg_circuit_add_source_wave(nsg_circuit* c, int is_voltage, int p, int n, int wave,
                                int nvalues, const double* values) {
    return guarded("nsg_circuit_add_source_wave", [&]() -> int {
        if (!c || nvalues < 0 || (nvalues && !values))
            return fail(NSG_ERR_INVALID, "bad arguments");
        if (wave != NSG_WAVE_DC && wave != NSG_WAVE_PULSE && wave != NSG_WAVE_PWL)
            return fail(NSG_ERR_INVALID, "nsg_circuit_add_source_wave: unknown waveform");
        c->c.add_source_wave(is_voltage != 0, p, n, static_cast<nsg::Wave>(wave),
                             std::vector<double>(values, values + nvalues));
        return NSG_OK;
    });
}

int nsg_circuit_add_mos1_model(nsg_circuit* c, int type, int nparams, const char* const* keys,
                               const double* values, int* model_out) {
    return guarded("nsg_circuit_add_mos1_model", [&]() -> int {
        if (!c || nparams < 0 || (nparams && (!keys || !values)) || !model_out)
            return fail(NSG_ERR_INVALID, "bad arguments");
        nsg::Mos1Card card;
        card.type = type;
        for (int i = 0; i < nparams; ++i) {
            if (!keys[i]) return fail(NSG_ERR_INVALID, "nsg_circuit_add_mos1_model: null key");
            card.params.emplace_back(keys[i], values[i]);
        }
        *model_out = c->c.add_mos1_model(card);
        return NSG_OK;
    });
}

int nsg_circuit_add_mosfet(nsg_circuit* c, int d, int g, int s, int b, int model, double w,
                           double l) {
    return guarded("nsg_circuit_add_mosfet", [&]() -> int {
        if (!c) return fail(NSG_ERR_INVALID, "null circuit");
        c->c.add_mosfet(d, g, s, b, model, w, l);
        return NSG_OK;
    });
}

int nsg_circuit_add_bsim4_model(nsg_circuit* c, int type, int nparams, const char* const* keys,
                                const double* values, int* model_out) {
    return guarded("nsg_circuit_add_bsim4_model", [&]() -> int {
        if (!c || nparams < 0 || (nparams && (!keys || !values)) || !model_out)
            return fail(NSG_ERR_INVALID, "bad arguments");
        nsg::Bsim4Card card;
        card.type = type;
        for (int i = 0; i < nparams; ++i) {
            if (!keys[i]) return fail(NSG_ERR_INVALID, "nsg_circuit_add_bsim4_model: null key");
            card.params.emplace_back(keys[i], values[i]);
        }
        *model_out = c->c.add_bsim4_model(card);
        return NSG_OK;
    });
}

int nsg_circuit_add_bsim4(nsg_circuit* c, int d, int g, int s, int b, int model, double w,
                          double l, double delvto) {
    return guarded("nsg_circuit_add_bsim4", [&]() -> int {
        if (!c) return fail(NSG_ERR_INVALID, "null circuit");
        c->c.add_bsim4(d, g, s, b, model, w, l, delvto);
        return NSG_OK;
    });
}

int nsg_circuit_add_capacitors(nsg_circuit* c, int count, const int* a, const int* b,
                               const double* farads) {
    return guarded("nsg_circuit_add_capacitors", [&]() -> int {
        if (!c || count < 0 || (count && (!a || !b || !farads)))
            return fail(NSG_ERR_INVALID, "bad arguments");
        for (int i = 0; i < count; ++i) c->c.add_capacitor(a[i], b[i], farads[i], false, 0.0);
        return NSG_OK;
    });
}

int nsg_circuit_add_resistors(nsg_circuit* c, int count, const int* a, const int* b,
                              const double* ohms) {
    return guarded("nsg_circuit_add_resistors", [&]() -> int {
        if (!c || count < 0 || (count && (!a || !b || !ohms)))
            return fail(NSG_ERR_INVALID, "bad arguments");
        for (int i = 0; i < count; ++i) c->c.add_resistor(a[i], b[i], ohms[i]);
        return NSG_OK;
    });
}

int nsg_circuit_add_isources(nsg_circuit* c, int count, const int* p, const int* n,
                             const double* amps) {
    return guarded("nsg_circuit_add_isources", [&]() -> int {
        if (!c || count < 0 || (count && (!p || !n || !amps)))
            return fail(NSG_ERR_INVALID, "bad arguments");
        for (int i = 0; i < count; ++i) c->c.add_isource(p[i], n[i], amps[i]);
        return NSG_OK;
    });
}

int nsg_circuit_add_diodes(nsg_circuit* c, int count, const int* anode, const int* cathode,
                           const double* is, const double* n_emission) {
    return guarded("nsg_circuit_add_diodes", [&]() -> int {
        if (!c || count < 0 || (count && (!anode || !cathode || !is || !n_emission)))
            return fail(NSG_ERR_INVALID, "bad arguments");
        for (int i = 0; i < count; ++i) c->c.add_diode(anode[i], cathode[i], is[i], n_emission[i]);
        return NSG_OK;
    });
}

int nsg_circuit_finalize(nsg_circuit* c) {
    return guarded("nsg_circuit_finalize", [&]() -> int {
        if (!c) return fail(NSG_ERR_INVALID, "null circuit");
        c->c.finalize();
        return NSG_OK;
    });
}

int nsg_circuit_info(const nsg_circuit* c, int* num_vars, int* num_nodes, int* nnz,
                     int* num_params) {
    if (!c) return fail(NSG_ERR_INVALID, "nsg_circuit_info: null circuit");
    if (!c->c.finalized()) return fail(NSG_ERR_INVALID, "nsg_circuit_info: not finalized");
    if (num_vars) *num_vars = c->c.num_vars();
    if (num_nodes) *num_nodes = c->c.num_nodes();
    if (nnz) *nnz = c->c.nnz();
    if (num_params) *num_params = static_cast<int>(c->c.params().size());
    return NSG_OK;
}

int nsg_circuit_pattern(const nsg_circuit* c, int* col_ptr, int* row_idx) {
    if (!c || !c->c.finalized()) return fail(NSG_ERR_INVALID, "nsg_circuit_pattern: not finalized");
    if (col_ptr) std::memcpy(col_ptr, c->c.col_ptr().data(), sizeof(int) * c->c.col_ptr().size());
    if (row_idx) std::memcpy(row_idx, c->c.row_idx().data(), sizeof(int) * c->c.row_idx().size());
    return NSG_OK;
}

int nsg_circuit_params(const nsg_circuit* c, double* params) {
    if (!c || !params) return fail(NSG_ERR_INVALID, "nsg_circuit_params: null argument");
    std::memcpy(params, c->c.params().data(), sizeof(double) * c->c.params().size());
    return NSG_OK;
}

int nsg_circuit_param_count(const nsg_circuit* c, int* count) {
    if (!c || !count) return fail(NSG_ERR_INVALID, "nsg_circuit_param_count: null argument");
    *count = static_cast<int>(c->c.params().size());
    return NSG_OK;
}

int nsg_circuit_set_param(nsg_circuit* c, int index, double value) {
    if (!c || index < 0 || index >= static_cast<int>(c->c.params().size()))
        return fail(NSG_ERR_INVALID, "nsg_circuit_set_param: bad arguments");
    c->c.params_mut()[index] = value;
    return NSG_OK;
}

int nsg_step_values(double start, double stop, double step, int cap, double* values, int* count) {
    if (!count || !(step != 0.0) || !std::isfinite(start) || !std::isfinite(stop) ||
        !std::isfinite(step) || cap < 0 || (cap > 0 && !values))
        return fail(NSG_ERR_INVALID, "nsg_step_values: bad arguments");
    // Simulator::run_step_sweep's loop: accumulate the step, stop a
    // thousandth of a step past `stop`.
    const int direction = (step > 0) ? 1 : -1;
    const double slack = std::abs(step) * 0.001;
    int k = 0;
    for (double v = start; direction > 0 ? v <= stop + slack : v >= stop - slack; v += step) {
        if (k >= (1 << 24)) return fail(NSG_ERR_INVALID, "nsg_step_values: too many steps");
        if (k < cap) values[k] = v;
        ++k;
    }
    *count = k;
    if (cap == 0) return NSG_OK;  // a size query
    return k <= cap ? NSG_OK : fail(NSG_ERR_INVALID, "nsg_step_values: capacity too small");
}

int nsg_circuit_initial_matrix(const nsg_circuit* c, double gmin, double* values, double* rhs) {
    return guarded("nsg_circuit_initial_matrix", [&]() -> int {
        if (!c || !c->c.finalized()) return fail(NSG_ERR_INVALID, "not finalized");
        std::vector<double> a, r;
        c->c.initjct_values(a, r, gmin);
        if (values) std::memcpy(values, a.data(), sizeof(double) * a.size());
        if (rhs) std::memcpy(rhs, r.data(), sizeof(double) * r.size());
        return NSG_OK;
    });
}

int nsg_circuit_eval_matrix(const nsg_circuit* c, int mode, const double* x, const double* ctx,
                            int order, int method, double gmin, double reltol, double abstol,
                            double* states, double* mos_rec, double* values, double* rhs) {
    return guarded("nsg_circuit_eval_matrix", [&]() -> int {
        if (!c || !c->c.finalized()) return fail(NSG_ERR_INVALID, "not finalized");
        if (!x || !ctx || !states || !mos_rec)
            return fail(NSG_ERR_INVALID, "nsg_circuit_eval_matrix: null argument");
        const nsg::Mos1Integ ic{ctx[0], ctx[1], ctx[2], ctx[3], ctx[4], ctx[5], order, method};
        std::vector<double> a, r;
        c->c.eval_values(mode, x, ic, ctx[6], gmin, reltol, abstol, states, mos_rec, a, r);
        if (values) std::memcpy(values, a.data(), sizeof(double) * a.size());
        if (rhs) std::memcpy(rhs, r.data(), sizeof(double) * r.size());
        return NSG_OK;
    });
}

int nsg_circuit_state_count(const nsg_circuit* c) {
    if (!c || !c->c.finalized()) return fail(NSG_ERR_INVALID, "not finalized");
    return c->c.num_states();
}

int nsg_dc_batch_create(int count, nsg_circuit* const* circuits, int symbolic, int threads,
                        nsg_dc_batch** out) {
    return guarded("nsg_dc_batch_create", [&]() -> int {
        if (!out || count <= 0 || !circuits)
            return fail(NSG_ERR_INVALID, "nsg_dc_batch_create: bad arguments");
        if (symbolic != NSG_SYMBOLIC_PER_INSTANCE && symbolic != NSG_SYMBOLIC_PER_PATTERN)
            return fail(NSG_ERR_INVALID, "nsg_dc_batch_create: unknown symbolic mode");
        *out = nullptr;
        for (int i = 0; i < count; ++i)
            if (!circuits[i] || !circuits[i]->c.finalized())
                return fail(NSG_ERR_INVALID, "nsg_dc_batch_create: circuit not finalized");
        auto b = std::make_unique<nsg_dc_batch>();
        b->count = count;
        if (threads <= 0) threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));

        // Symbolic phase on the first-iteration (INITJCT) matrix, as the
        // reference's first NeoSolver::numeric in newton_solve sees it.
        std::vector<int> rep(count);  // instance whose ordering instance i uses
        if (symbolic == NSG_SYMBOLIC_PER_PATTERN) {
            std::map<std::pair<std::vector<int32_t>, std::vector<int32_t>>, int> first;
            for (int i = 0; i < count; ++i) {
                const auto& c = circuits[i]->c;
                auto key = std::make_pair(c.col_ptr(), c.row_idx());
                rep[i] = first.emplace(std::move(key), i).first->second;
            }
        } else {
            for (int i = 0; i < count; ++i) rep[i] = i;
        }
        std::vector<int> todo;
        for (int i = 0; i < count; ++i)
            if (rep[i] == i) todo.push_back(i);
        std::vector<std::unique_ptr<nsg_topology>> ordered(count);
        std::vector<int> rcs(count, NSG_OK);
        parallel_for(static_cast<int>(todo.size()), threads, [&](int k) {
            const int i = todo[k];
            const auto& c = circuits[i]->c;
            std::vector<double> a, r;
            c.initjct_values(a, r, b->opt.gmin);
            rcs[i] = order_topology(c.num_vars(), c.nnz(), c.col_ptr().data(), c.row_idx().data(),
                                    a.data(), b->opt.diag_gmin, ordered[i],
                                    select_solver(c.num_vars(), c.is_linear()));
        });
        for (int i : todo)
            if (rcs[i] != NSG_OK)
                return fail(rcs[i], "nsg_dc_batch_create: symbolic phase failed for instance " +
                                        std::to_string(i));
        // Share identical symbolic results between instances.
        std::vector<int> topo_of(count, -1);
        for (int i : todo) {
            for (size_t t = 0; t < b->topos.size(); ++t)
                if (b->topos[t]->plan.n == ordered[i]->plan.n &&
                    same_plan(b->topos[t]->plan, ordered[i]->plan)) {
                    topo_of[i] = static_cast<int>(t);
                    break;
                }
            if (topo_of[i] < 0) {
                topo_of[i] = static_cast<int>(b->topos.size());
                b->topos.push_back(std::move(ordered[i]));
            }
        }
        for (int i = 0; i < count; ++i) topo_of[i] = topo_of[rep[i]];

        // Device plans, programs, descriptors, workspace.
        std::vector<int32_t> lu_pool, prog;
        std::vector<nsg::PlanDesc> plans;
        for (const auto& t : b->topos) {
            if (!t->plan.has_update_map)
                throw std::invalid_argument("circuit too large for the batched Newton kernels "
                                            "(its factorization has no update map)");
            plans.push_back(make_plan_desc(t->plan, lu_pool));
            b->max_col = std::max(b->max_col, t->plan.max_col);
            b->max_n = std::max(b->max_n, t->plan.n);
        }
        std::vector<nsg::DcDesc> descs(count);
        b->param_off.assign(count + 1, 0);
        b->sol_off.assign(count + 1, 0);
        int64_t work = 0;
        for (int i = 0; i < count; ++i) {
            const auto& c = circuits[i]->c;
            const auto& p = b->topos[topo_of[i]]->plan;
            nsg::DcDesc& d = descs[i];
            fill_instance(d, c, p, prog, work);
            place_dcsave(d, work);
            d.index = i;
            d.plan = topo_of[i];
            d.param_off = b->param_off[i];
            d.sol_off = b->sol_off[i];
            b->param_off[i + 1] = b->param_off[i] + static_cast<int64_t>(c.params().size());
            b->sol_off[i + 1] = b->sol_off[i] + c.num_vars();
            b->host_params.insert(b->host_params.end(), c.params().begin(), c.params().end());
            b->inst_n.push_back(p.n);
            b->inst_nnz.push_back(p.nnz_a);
            b->inst_nnz_lu.push_back(p.nnz_lu);
            b->inst_updates.push_back(p.updates);
            b->updates += p.updates;
            b->nnz_lu += p.nnz_lu;
            b->nnz += p.nnz_a;
            b->n += p.n;
        }
        // Launch the most expensive instances first so the grid's tail is
        // made of small ones.
        std::stable_sort(descs.begin(), descs.end(), [&](const nsg::DcDesc& x, const nsg::DcDesc& y) {
            return b->inst_updates[x.index] > b->inst_updates[y.index];
        });
        const size_t smem = nsg::dc_smem_bytes(b->max_col, b->max_n);
        if (smem > 200 * 1024)
            return fail(NSG_ERR_INVALID, "nsg_dc_batch_create: instance too large for the "
                                         "shared-memory refactor (longest LU column " +
                                         std::to_string(b->max_col) + ")");
        b->desc_pos.assign(count, 0);
        for (int k = 0; k < count; ++k) b->desc_pos[descs[k].index] = k;
        b->topo_of = topo_of;
        b->work_size = b->work_cap = work;
        cudaError_t e;
        if ((e = upload(&b->d_lu_pool, lu_pool.data(), lu_pool.size())) != cudaSuccess ||
            (e = upload(&b->d_plans, plans.data(), plans.size())) != cudaSuccess ||
            (e = upload(&b->d_prog, prog.data(), prog.size())) != cudaSuccess ||
            (e = upload(&b->d_descs, descs.data(), descs.size())) != cudaSuccess ||
            (e = upload<double>(&b->d_work, nullptr, static_cast<size_t>(work))) != cudaSuccess ||
            (e = upload(&b->d_params, b->host_params.data(), b->host_params.size())) != cudaSuccess ||
            (e = upload<nsg::DcCtl>(&b->d_ctl, nullptr, count)) != cudaSuccess ||
            (e = upload<int32_t>(&b->d_subset, nullptr, count)) != cudaSuccess)
            return cuda_fail("nsg_dc_batch_create", e);
        b->descs = std::move(descs);
        *out = b.release();
        return NSG_OK;
    });
}

void nsg_dc_batch_free(nsg_dc_batch* b) { delete b; }

int nsg_dc_batch_layout(const nsg_dc_batch* b, long long* param_offsets,
                        long long* solution_offsets) {
    if (!b) return fail(NSG_ERR_INVALID, "nsg_dc_batch_layout: null batch");
    const size_t bytes = sizeof(long long) * (b->count + 1);
    if (param_offsets) std::memcpy(param_offsets, b->param_off.data(), bytes);
    if (solution_offsets) std::memcpy(solution_offsets, b->sol_off.data(), bytes);
    return NSG_OK;
}

int nsg_dc_batch_stats(const nsg_dc_batch* b, long long* n, long long* nnz, long long* nnz_lu,
                       long long* updates, int* distinct_topologies) {
    if (!b) return fail(NSG_ERR_INVALID, "nsg_dc_batch_stats: null batch");
    if (n) *n = b->n;
    if (nnz) *nnz = b->nnz;
    if (nnz_lu) *nnz_lu = b->nnz_lu;
    if (updates) *updates = b->updates;
    if (distinct_topologies) *distinct_topologies = static_cast<int>(b->topos.size());
    return NSG_OK;
}

int nsg_dc_batch_instance_stats(const nsg_dc_batch* b, long long* n, long long* nnz,
                                long long* nnz_lu, long long* updates) {
    if (!b) return fail(NSG_ERR_INVALID, "nsg_dc_batch_instance_stats: null batch");
    const size_t bytes = sizeof(long long) * b->count;
    if (n) std::memcpy(n, b->inst_n.data(), bytes);
    if (nnz) std::memcpy(nnz, b->inst_nnz.data(), bytes);
    if (nnz_lu) std::memcpy(nnz_lu, b->inst_nnz_lu.data(), bytes);
    if (updates) std::memcpy(updates, b->inst_updates.data(), bytes);
    return NSG_OK;
}

int nsg_dc_batch_set_options(nsg_dc_batch* b, double reltol, double vntol, double abstol,
                             double gmin, int max_iter) {
    if (!b || max_iter <= 0) return fail(NSG_ERR_INVALID, "nsg_dc_batch_set_options: bad arguments");
    b->opt.reltol = reltol;
    b->opt.vntol = vntol;
    b->opt.abstol = abstol;
    b->opt.gmin = gmin;
    b->opt.max_iter = max_iter;
    b->drop_graph();  // the captured launch holds the options by value
    return NSG_OK;
}

int nsg_dc_batch_set_first_aid(nsg_dc_batch* b, int aid) {
    if (!b || aid < nsg::kAidDirect || aid > nsg::kAidPseudoTransient)
        return fail(NSG_ERR_INVALID, "nsg_dc_batch_set_first_aid: bad arguments");
    b->opt.first_aid = aid;
    b->drop_graph();
    return NSG_OK;
}

int nsg_dc_batch_set_reorder(nsg_dc_batch* b, int enable) {
    if (!b) return fail(NSG_ERR_INVALID, "nsg_dc_batch_set_reorder: null batch");
    b->reorder = enable != 0;
    return NSG_OK;
}

int nsg_dc_batch_set_graph(nsg_dc_batch* b, int enable) {
    return guarded("nsg_dc_batch_set_graph", [&]() -> int {
        if (!b) return fail(NSG_ERR_INVALID, "nsg_dc_batch_set_graph: null batch");
        b->use_graph = enable != 0;
        b->drop_graph();
        if (b->use_graph && !b->cap_stream) {
            const cudaError_t e = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
            if (e != cudaSuccess) return cuda_fail("nsg_dc_batch_set_graph", e);
        }
        return NSG_OK;
    });
}

int nsg_dc_batch_set_row_maps(nsg_dc_batch* b, int enable) {
    if (!b) return fail(NSG_ERR_INVALID, "nsg_dc_batch_set_row_maps: null batch");
    b->row_maps = enable != 0;
    b->drop_graph();
    return NSG_OK;
}

int nsg_dc_batch_graph_launches(const nsg_dc_batch* b, long long* count) {
    if (!b || !count) return fail(NSG_ERR_INVALID, "nsg_dc_batch_graph_launches: null argument");
    *count = b->graph_launches;
    return NSG_OK;
}

int nsg_dc_batch_reorders(const nsg_dc_batch* b, long long* count) {
    if (!b || !count) return fail(NSG_ERR_INVALID, "nsg_dc_batch_reorders: null argument");
    *count = b->reorders;
    return NSG_OK;
}

int nsg_dc_batch_engines(const nsg_dc_batch* b, int* engine) {
    if (!b || !engine) return fail(NSG_ERR_INVALID, "nsg_dc_batch_engines: null argument");
    for (int i = 0; i < b->count; ++i)
        engine[i] = b->topos[b->topo_of[i]]->plan.kind == nsg::kPlanKindAmdLu
                        ? NSG_SOLVER_AMDLU
                        : NSG_SOLVER_MARKOWITZ;
    return NSG_OK;
}

int nsg_dc_batch_methods(const nsg_dc_batch* b, int* method, int* solves) {
    if (!b) return fail(NSG_ERR_INVALID, "nsg_dc_batch_methods: null batch");
    std::vector<nsg::DcCtl> ctl(b->count);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess)
        e = cudaMemcpy(ctl.data(), b->d_ctl, sizeof(nsg::DcCtl) * b->count, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail("nsg_dc_batch_methods", e);
    for (int i = 0; i < b->count; ++i) {
        if (method) method[i] = ctl[i].method;
        if (solves) solves[i] = ctl[i].solves;
    }
    return NSG_OK;
}

int nsg_dc_batch_adjoint(nsg_dc_batch* b, const double* d_params, const double* d_solutions,
                         const double* d_cotangent, double* d_grads, int* d_status, void* stream) {
    if (!b || !d_solutions || !d_cotangent || !d_grads || !d_status)
        return fail(NSG_ERR_INVALID, "nsg_dc_batch_adjoint: null argument");
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(d_grads, 0, sizeof(double) * b->param_off[b->count], st);
    if (e == cudaSuccess)
        e = nsg::launch_dc_adjoint(b->d_plans, b->d_lu_pool, b->d_descs, b->count, b->d_prog,
                                   d_params ? d_params : b->d_params, b->d_work, d_solutions,
                                   d_cotangent, d_grads, d_status, b->opt, b->max_col, b->max_n,
                                   st);
    return e == cudaSuccess ? NSG_OK : cuda_fail("nsg_dc_batch_adjoint", e);
}

int nsg_dc_batch_run(nsg_dc_batch* b, const double* d_params, double* d_solutions, int* d_status,
                     int* d_iterations, void* stream) {
    return guarded("nsg_dc_batch_run", [&]() -> int {
        if (!b || !d_solutions || !d_status || !d_iterations)
            return fail(NSG_ERR_INVALID, "nsg_dc_batch_run: null argument");
        const cudaStream_t st = static_cast<cudaStream_t>(stream);
        const double* params = d_params ? d_params : b->d_params;
        if (b->row_maps) {
            // warps per CTA of newton_dc_kernel (16), max_n words each
            const int64_t words = int64_t{b->count} * 16 * b->max_n;
            if (words > b->rmap_cap) {
                b->drop_graph();
                cudaFree(b->d_rmap);
                b->d_rmap = nullptr;
                b->rmap_cap = 0;
                const cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&b->d_rmap),
                                                 sizeof(int32_t) * static_cast<size_t>(words));
                if (e != cudaSuccess) return cuda_fail("nsg_dc_batch_run", e);
                b->rmap_cap = words;
            }
        }
        int32_t* rmaps = b->row_maps ? b->d_rmap : nullptr;
        auto first_launch = [&](cudaStream_t s) -> cudaError_t {
            cudaError_t r = cudaMemsetAsync(b->d_ctl, 0, sizeof(nsg::DcCtl) * b->count, s);
            if (r == cudaSuccess)
                r = nsg::launch_newton_dc(b->d_plans, b->d_lu_pool, b->d_descs, nullptr, b->count,
                                          b->d_prog, params, b->d_work, d_solutions, d_status,
                                          d_iterations, b->d_ctl, b->opt, b->max_col, b->max_n,
                                          max_stage_len(b->descs), rmaps, s);
            return r;
        };
        cudaError_t e = cudaSuccess;
        const void* key[4] = {params, d_solutions, d_status, d_iterations};
        if (b->use_graph && b->graph && std::equal(key, key + 4, b->graph_key)) {
            e = cudaGraphLaunch(b->graph, st);
            ++b->graph_launches;
        } else if (b->use_graph && b->plain_launches > 0 && b->cap_stream) {
            // Capture the launch on the batch's own stream (the caller's may
            // be the legacy default stream, which cannot be captured), then
            // replay it on the caller's stream.
            b->drop_graph();
            cudaGraph_t g = nullptr;
            e = cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                const cudaError_t le = first_launch(b->cap_stream);
                e = cudaStreamEndCapture(b->cap_stream, &g);
                if (e == cudaSuccess) e = le;
            }
            if (e == cudaSuccess) e = cudaGraphInstantiate(&b->graph, g, 0);
            if (g) cudaGraphDestroy(g);
            if (e == cudaSuccess) {
                std::copy(key, key + 4, b->graph_key);
                e = cudaGraphLaunch(b->graph, st);
                ++b->graph_launches;
            } else {
                b->drop_graph();
            }
        } else {
            // plain launch (also the first of a graph-enabled batch, which
            // configures the kernel before any capture)
            e = first_launch(st);
            ++b->plain_launches;
        }
        if (e != cudaSuccess) return cuda_fail("nsg_dc_batch_run", e);
        if (!b->reorder) return NSG_OK;
        // Instances whose pivots failed re-validation: re-order on the host
        // (NeoSolver::numeric's order_and_factor from the failing step) and
        // resume them on the device.
        std::vector<int> status(b->count);
        for (int round = 0; round < 64; ++round) {
            if ((e = cudaStreamSynchronize(st)) != cudaSuccess ||
                (e = cudaMemcpy(status.data(), d_status, sizeof(int) * b->count,
                                cudaMemcpyDeviceToHost)) != cudaSuccess)
                return cuda_fail("nsg_dc_batch_run", e);
            std::vector<int32_t> subset;
            for (int i = 0; i < b->count; ++i) {
                if (status[i] != NSG_REORDER) continue;
                nsg::DcDesc& d = b->descs[b->desc_pos[i]];
                std::vector<double> a(d.nnz);
                nsg::DcCtl ctl;
                if ((e = cudaMemcpy(a.data(), b->d_work + d.a_off, sizeof(double) * d.nnz,
                                    cudaMemcpyDeviceToHost)) != cudaSuccess ||
                    (e = cudaMemcpy(&ctl, b->d_ctl + i, sizeof ctl, cudaMemcpyDeviceToHost)) !=
                        cudaSuccess)
                    return cuda_fail("nsg_dc_batch_run", e);
                int topo = 0;
                const int rc = reorder_instance(b->topos, b->topo_of[i], a.data(),
                                                ctl.numeric_diag_gmin, &topo);
                if (rc != NSG_OK) continue;  // stays NSG_REORDER: the host could not re-order
                b->topo_of[i] = topo;
                d.plan = topo;
                place_lu_workspace(d, b->topos[topo]->plan, b->work_size);
                subset.push_back(b->desc_pos[i]);
                ++b->reorders;
            }
            if (subset.empty()) break;
            b->drop_graph();  // plans and workspace move
            int rc = refresh_plans(b->topos, &b->d_lu_pool, &b->d_plans, &b->max_col, &b->max_n);
            if (rc != NSG_OK) return rc;
            if (nsg::dc_smem_bytes(b->max_col, b->max_n) > 200 * 1024)
                return fail(NSG_ERR_INVALID, "nsg_dc_batch_run: re-ordered instance too large "
                                             "for the shared-memory refactor");
            if ((e = grow_workspace(&b->d_work, &b->work_cap, b->work_size)) != cudaSuccess ||
                (e = cudaMemcpy(b->d_descs, b->descs.data(), sizeof(nsg::DcDesc) * b->count,
                                cudaMemcpyHostToDevice)) != cudaSuccess ||
                (e = cudaMemcpy(b->d_subset, subset.data(), sizeof(int32_t) * subset.size(),
                                cudaMemcpyHostToDevice)) != cudaSuccess ||
                (e = nsg::launch_newton_dc(b->d_plans, b->d_lu_pool, b->d_descs, b->d_subset,
                                           static_cast<int>(subset.size()), b->d_prog, params,
                                           b->d_work, d_solutions, d_status, d_iterations,
                                           b->d_ctl, b->opt, b->max_col, b->max_n,
                                           max_stage_len(b->descs), rmaps, st)) !=
                    cudaSuccess)
                return cuda_fail("nsg_dc_batch_run", e);
        }
        return NSG_OK;
    });
}

}  // extern "C"
