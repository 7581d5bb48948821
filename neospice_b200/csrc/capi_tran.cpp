// C ABI of the batched transient analysis (include/nsgpu.h).
#include "capi_internal.hpp"

#include "host/circuit.hpp"
#include "kernels/mos1_charge_adjoint.cuh"
#include "kernels/mos1_model.cuh"
#include "kernels/tran_device.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <thread>

namespace nsg {
cudaError_t launch_transient(const PlanDesc* plans, const int32_t* lu_pool, const DcDesc* descs,
                             const TranDesc* tdescs, const int32_t* subset, int count,
                             const int32_t* prog, const double* params_dc,
                             const double* params_tran, double* work, const double* bps,
                             const int32_t* probes, double* times, double* values,
                             int32_t* npoints, int32_t* status, int32_t* stats, TranCtl* ctls,
                             const TranOptions& o, const TranShape& shape,
                             StepRecord* rec_steps, double* rec_x0, cudaStream_t stream);
size_t tran_smem_bytes(int max_col, int max_n);
struct AdjDesc {
    int32_t n_steps, every, probe, n_ckpt;
    int64_t rec_off, x0_off, ws_off, ckpt_len;
};
cudaError_t launch_tran_adjoint(const PlanDesc* plans, const int32_t* lu_pool, const DcDesc* descs,
                                const TranDesc* tdescs, const AdjDesc* adescs, int count,
                                const int32_t* prog, const double* params_dc,
                                const double* params_tran, double* work, double* adj_ws,
                                const StepRecord* recs, const double* times, const double* rec_x0,
                                const double* targets, double weight, double* grads, double* loss,
                                int32_t* status, const NewtonOptions& opt, int max_iter,
                                int max_col, int max_n, cudaStream_t stream);
}  // namespace nsg

using namespace nsg_internal;

struct nsg_tran_batch {
    int count = 0;
    nsg::TranOptions opt{};
    std::vector<std::unique_ptr<nsg_topology>> topos;
    std::vector<nsg::DcDesc> descs;      // launch order = instance order
    std::vector<nsg::TranDesc> tdescs;
    std::vector<std::vector<int32_t>> col_ptr, row_idx;  // per-instance pattern
    std::vector<int> solver;  // per-instance engine (NSG_SOLVER_*), as make_solver picks it
    int max_col = 0, max_n = 0;
    int force_threads = 0, force_blocks = 0;  // nsg_tran_batch_set_shape
    // Descriptors and workspace size as created: every run starts from them
    // (the DC plan ordered on the first DC matrix, no transient plan yet),
    // as the reference's solve_transient starts from fresh solvers.
    std::vector<nsg::DcDesc> descs0;
    std::vector<nsg::TranDesc> tdescs0;
    int64_t work_size0 = 0;
    int64_t work_size = 0, work_cap = 0;
    long long orderings = 0;
    // Host orderings made by earlier runs, per instance: the request (first
    // ordering or re-ordering from plan `from`, diag_gmin), the matrix it was
    // made from and the topology it gave.  The ordering is a deterministic
    // function of these, so a run that stops with a bit-identical request
    // takes the topology without ordering again (a re-run with unchanged
    // parameters re-orders nothing).
    struct OrderMemo {
        int need, from;
        double diag_gmin;
        std::vector<double> a;
        int topo;
    };
    std::vector<std::vector<OrderMemo>> memo;
    int32_t* d_lu_pool = nullptr;
    nsg::PlanDesc* d_plans = nullptr;
    int32_t* d_prog = nullptr;
    nsg::DcDesc* d_descs = nullptr;
    nsg::TranDesc* d_tdescs = nullptr;
    double* d_work = nullptr;
    double* d_params_dc = nullptr;
    double* d_params_tran = nullptr;
    double* d_bps = nullptr;
    int32_t* d_probes = nullptr;
    double* d_times = nullptr;
    double* d_values = nullptr;
    int32_t* d_npoints = nullptr;
    int32_t* d_status = nullptr;
    int32_t* d_stats = nullptr;
    nsg::TranCtl* d_ctl = nullptr;
    int32_t* d_subset = nullptr;
    // Adjoint: recording of the forward run's steps and operating points,
    // the replay's Newton options, whether each circuit's devices are ones
    // the adjoint covers (no BSIM4v7), and its workspace.
    bool record = false, recorded = false;
    nsg::StepRecord* d_rec = nullptr;
    double* d_x0 = nullptr;
    std::vector<char> adjoint_ok;
    std::vector<int64_t> param_count;
    nsg::NewtonOptions adj_opt{1e-3, 1e-6, 1e-12, 1e-12, 0.0, 100, nsg::kAidDirect};
    int adj_max_iter = 100;
    double* d_adj_ws = nullptr;
    int64_t adj_ws_cap = 0;
    nsg::AdjDesc* d_adescs = nullptr;
    ~nsg_tran_batch() {
        cudaFree(d_rec);
        cudaFree(d_x0);
        cudaFree(d_adj_ws);
        cudaFree(d_adescs);
        for (void* p : {static_cast<void*>(d_lu_pool), static_cast<void*>(d_plans),
                        static_cast<void*>(d_prog), static_cast<void*>(d_descs),
                        static_cast<void*>(d_tdescs), static_cast<void*>(d_work),
                        static_cast<void*>(d_params_dc), static_cast<void*>(d_params_tran),
                        static_cast<void*>(d_bps), static_cast<void*>(d_probes),
                        static_cast<void*>(d_times), static_cast<void*>(d_values),
                        static_cast<void*>(d_npoints), static_cast<void*>(d_status),
                        static_cast<void*>(d_stats), static_cast<void*>(d_ctl),
                        static_cast<void*>(d_subset)})
            cudaFree(p);
    }
};

namespace {

// Launch shape of a transient batch (nsg::TranShape).
nsg::TranShape tran_shape(const nsg_tran_batch& b) {
    nsg::TranShape sh{b.max_col, b.max_n, max_stage_len(b.descs), 0, 0, 0,
                      b.force_threads, b.force_blocks};
    for (const auto& t : b.topos) {
        sh.max_small_lu = std::max(sh.max_small_lu, t->plan.nnz_lu + t->plan.n);
        sh.max_plan_words = std::max<int64_t>(sh.max_plan_words, t->plan.device_words());
    }
    for (const auto& d : b.descs)
        sh.max_devices = std::max({sh.max_devices, d.n_mos, d.n_diodes, d.n_caps, d.n_srcs});
    return sh;
}

}  // namespace

namespace {

// TimeStepController::add_source_breakpoint (src/core/timestep.cpp:105-127)
// for HARD breakpoints, in insertion order; returns the sorted set.
std::vector<double> controller_breakpoints(const std::vector<double>& raw, double tstop,
                                           double max_step) {
    const double min_break = (max_step > 0.0) ? 5e-5 * max_step : 0.0;
    std::vector<double> set;  // sorted, unique
    for (double t : raw) {
        if (!(t > 0.0 && t <= tstop)) continue;
        if (min_break > 0.0) {
            auto lb = std::lower_bound(set.begin(), set.end(), t - min_break);
            if (lb != set.end() && *lb <= t + min_break) continue;
        }
        auto it = std::lower_bound(set.begin(), set.end(), t);
        if (it == set.end() || *it != t) set.insert(it, t);
    }
    return set;
}

}  // namespace

extern "C" {

int nsg_tran_batch_create(int count, nsg_circuit* const* circuits, double tstep, double tstop,
                          int max_points, int nprobe, const int* probes, int threads,
                          nsg_tran_batch** out) {
    return guarded("nsg_tran_batch_create", [&]() -> int {
        if (!out || count <= 0 || !circuits || !(tstep > 0.0) || !(tstop > 0.0) ||
            max_points < 1 || nprobe < 1 || !probes)
            return fail(NSG_ERR_INVALID, "nsg_tran_batch_create: bad arguments");
        *out = nullptr;
        for (int i = 0; i < count; ++i) {
            if (!circuits[i] || !circuits[i]->c.finalized())
                return fail(NSG_ERR_INVALID, "nsg_tran_batch_create: circuit not finalized");
            for (int j = 0; j < nprobe; ++j)
                if (probes[j] < 0 || probes[j] >= circuits[i]->c.num_vars())
                    return fail(NSG_ERR_INVALID, "nsg_tran_batch_create: probe out of range");
        }
        auto b = std::make_unique<nsg_tran_batch>();
        b->count = count;
        if (threads <= 0) threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
        auto& o = b->opt;
        o.nopt = nsg::NewtonOptions{1e-3, 1e-6, 1e-12, 1e-12, 0.0, 100, nsg::kAidDirect};
        o.tstep = tstep;
        o.tstop = tstop;
        // transient.cpp:818-821: maxStep = min(tstep, tstop/50), dt_min = maxStep*1e-11
        const double max_step = std::min(tstep, tstop / 50.0);
        o.dt_max = max_step;
        o.dt_min = max_step * 1e-11;
        o.trtol = 7.0;
        o.chgtol = 1e-14;
        o.xmu = 0.5;
        o.restart_scale = 0.1;
        o.itl4 = 50;
        o.use_gear = 0;
        o.max_points = max_points;
        o.nprobe = nprobe;

        // Per instance: parameters with PULSE defaults resolved, breakpoints,
        // the initial dt, and the DC solver's ordering on the first DC Newton
        // matrix.  The transient solver is ordered later, on the first
        // transient iteration's matrix as the device computes it (the
        // reference creates two solvers, each ordered on its first matrix).
        std::vector<std::vector<double>> ptran(count), bps(count);
        std::vector<double> dt0(count);
        b->solver.resize(count);
        for (int i = 0; i < count; ++i) {
            const auto& c = circuits[i]->c;
            b->solver[i] = select_solver(c.num_vars(), c.is_linear());
            ptran[i] = c.resolved_params(tstep, tstop);
            bps[i] = controller_breakpoints(c.source_breakpoints(ptran[i], tstop), tstop, max_step);
            double dt = std::min(tstop / 100.0, tstep) / 10.0;  // transient.cpp:851
            const double gap = bps[i].empty() ? tstop : bps[i][0];
            if (gap < tstop) {
                dt = std::min(dt, 0.1 * std::min(tstop / 50.0, gap));
                dt /= 10;
                dt = std::max(dt, o.dt_min * 2.0);
            }
            dt0[i] = dt;
        }
        std::vector<std::unique_ptr<nsg_topology>> ord_dc(count);
        std::vector<int> rc_dc(count, NSG_OK);
        std::atomic<int> next{0};
        std::vector<std::thread> pool;
        for (int t = 0; t < std::min(threads, count); ++t)
            pool.emplace_back([&] {
                for (int i; (i = next.fetch_add(1)) < count;) {
                    const auto& c = circuits[i]->c;
                    std::vector<double> a, r;
                    c.initjct_values(a, r, o.nopt.gmin);
                    rc_dc[i] = order_topology(c.num_vars(), c.nnz(), c.col_ptr().data(),
                                              c.row_idx().data(), a.data(), 0.0, ord_dc[i],
                                              b->solver[i]);
                }
            });
        for (auto& th : pool) th.join();
        for (int i = 0; i < count; ++i)
            if (rc_dc[i] != NSG_OK)
                return fail(NSG_SINGULAR, "nsg_tran_batch_create: symbolic phase failed for "
                                          "instance " + std::to_string(i));
        std::vector<int> plan_dc(count);
        for (int i = 0; i < count; ++i) plan_dc[i] = intern_topology(b->topos, std::move(ord_dc[i]));

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
        b->descs.resize(count);
        b->tdescs.resize(count);
        std::vector<double> params_dc, params_tran, all_bps;
        int64_t work = 0, param_off = 0, x0_off = 0;
        for (int i = 0; i < count; ++i) {
            const auto& c = circuits[i]->c;
            // The adjoint covers resistors, capacitors, sources, diodes and
            // level-1 MOSFETs with their Meyer and junction charges; not
            // BSIM4v7 devices.
            b->adjoint_ok.push_back(c.has_bsim4() ? 0 : 1);
            b->param_count.push_back(static_cast<int64_t>(c.params().size()));
            nsg::DcDesc& d = b->descs[i];
            fill_instance(d, c, b->topos[plan_dc[i]]->plan, prog, work);
            d.index = i;
            d.plan = plan_dc[i];
            d.param_off = param_off;
            d.sol_off = 0;
            param_off += static_cast<int64_t>(c.params().size());
            params_dc.insert(params_dc.end(), c.params().begin(), c.params().end());
            params_tran.insert(params_tran.end(), ptran[i].begin(), ptran[i].end());
            nsg::TranDesc& t = b->tdescs[i];
            t.tran_plan = -1;
            t.n_bps = static_cast<int32_t>(bps[i].size());
            t.bp_off = static_cast<int64_t>(all_bps.size());
            all_bps.insert(all_bps.end(), bps[i].begin(), bps[i].end());
            t.out_off = static_cast<int64_t>(i) * max_points;
            t.hist_off = work;
            work += (3 * static_cast<int64_t>(c.num_vars()) + 3) & ~int64_t{3};
            d.stage_len = work - d.x_off;
            place_dcsave(d, work);
            t.dt0 = dt0[i];
            t.x0_off = x0_off;
            x0_off += c.num_vars();
            b->col_ptr.push_back(c.col_ptr());
            b->row_idx.push_back(c.row_idx());
        }
        b->work_size = b->work_cap = work;
        b->descs0 = b->descs;
        b->tdescs0 = b->tdescs;
        b->work_size0 = work;
        const size_t smem = nsg::tran_smem_bytes(b->max_col, b->max_n);
        if (smem > 200 * 1024)
            return fail(NSG_ERR_INVALID, "nsg_tran_batch_create: instance too large for the "
                                         "shared-memory refactor");
        std::vector<int32_t> pr(probes, probes + nprobe);
        const size_t nout = static_cast<size_t>(count) * max_points;
        cudaError_t e;
        if ((e = upload(&b->d_lu_pool, lu_pool.data(), lu_pool.size())) != cudaSuccess ||
            (e = upload(&b->d_plans, plans.data(), plans.size())) != cudaSuccess ||
            (e = upload(&b->d_prog, prog.data(), prog.size())) != cudaSuccess ||
            (e = upload(&b->d_descs, b->descs.data(), b->descs.size())) != cudaSuccess ||
            (e = upload(&b->d_tdescs, b->tdescs.data(), b->tdescs.size())) != cudaSuccess ||
            (e = upload<double>(&b->d_work, nullptr, static_cast<size_t>(work))) != cudaSuccess ||
            (e = upload(&b->d_params_dc, params_dc.data(), params_dc.size())) != cudaSuccess ||
            (e = upload(&b->d_params_tran, params_tran.data(), params_tran.size())) != cudaSuccess ||
            (e = upload(&b->d_bps, all_bps.data(), all_bps.size())) != cudaSuccess ||
            (e = upload(&b->d_probes, pr.data(), pr.size())) != cudaSuccess ||
            (e = upload<double>(&b->d_times, nullptr, nout)) != cudaSuccess ||
            (e = upload<double>(&b->d_values, nullptr, nout * nprobe)) != cudaSuccess ||
            (e = upload<int32_t>(&b->d_npoints, nullptr, count)) != cudaSuccess ||
            (e = upload<int32_t>(&b->d_status, nullptr, count)) != cudaSuccess ||
            (e = upload<int32_t>(&b->d_stats, nullptr, 4 * static_cast<size_t>(count))) != cudaSuccess ||
            (e = upload<nsg::TranCtl>(&b->d_ctl, nullptr, count)) != cudaSuccess ||
            (e = upload<int32_t>(&b->d_subset, nullptr, count)) != cudaSuccess)
            return cuda_fail("nsg_tran_batch_create", e);
        *out = b.release();
        return NSG_OK;
    });
}

void nsg_tran_batch_free(nsg_tran_batch* b) { delete b; }

int nsg_tran_batch_set_shape(nsg_tran_batch* b, int threads, int blocks_per_sm) {
    if (!b) return fail(NSG_ERR_INVALID, "nsg_tran_batch_set_shape: null batch");
    const bool ok = (threads == 0 && blocks_per_sm == 0) ||
                    (threads == 128 && (blocks_per_sm == 0 || blocks_per_sm == 8)) ||
                    (threads == 256 && (blocks_per_sm == 0 || blocks_per_sm == 4)) ||
                    (threads == 512 && (blocks_per_sm == 0 || blocks_per_sm == 2));
    if (!ok) return fail(NSG_ERR_INVALID, "nsg_tran_batch_set_shape: unsupported shape");
    if (threads != 0 && threads != 512 && b->max_n > 128)
        return fail(NSG_ERR_INVALID, "nsg_tran_batch_set_shape: instances above 128 unknowns "
                                     "need 512-thread CTAs");
    b->force_threads = threads;
    b->force_blocks = blocks_per_sm;
    return NSG_OK;
}

int nsg_tran_batch_run(nsg_tran_batch* b, void* stream) {
    return guarded("nsg_tran_batch_run", [&]() -> int {
        if (!b) return fail(NSG_ERR_INVALID, "nsg_tran_batch_run: null batch");
        const cudaStream_t st = static_cast<cudaStream_t>(stream);
        auto launch = [&](const int32_t* subset, int n) {
            return nsg::launch_transient(b->d_plans, b->d_lu_pool, b->d_descs, b->d_tdescs, subset,
                                         n, b->d_prog, b->d_params_dc, b->d_params_tran, b->d_work,
                                         b->d_bps, b->d_probes, b->d_times, b->d_values,
                                         b->d_npoints, b->d_status, b->d_stats, b->d_ctl, b->opt,
                                         tran_shape(*b),
                                         b->record ? b->d_rec : nullptr,
                                         b->record ? b->d_x0 : nullptr, st);
        };
        b->recorded = false;
        // Start from the batch as created: the plans and LU regions a
        // previous run's re-orderings placed are not this run's (a reused
        // transient plan would also hand the DC phase an LU region sized for
        // another plan).
        b->descs = b->descs0;
        b->tdescs = b->tdescs0;
        b->work_size = b->work_size0;
        cudaError_t e = cudaMemcpy(b->d_descs, b->descs.data(), sizeof(nsg::DcDesc) * b->count,
                                   cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(b->d_tdescs, b->tdescs.data(), sizeof(nsg::TranDesc) * b->count,
                           cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemsetAsync(b->d_ctl, 0, sizeof(nsg::TranCtl) * b->count, st);
        if (e == cudaSuccess) e = launch(nullptr, b->count);
        if (e != cudaSuccess) return cuda_fail("nsg_tran_batch_run", e);
        // Instances stop for the host when a solver needs its first ordering
        // (the transient solver, on the first transient matrix) or a
        // re-ordering after a failed pivot re-validation; each is ordered
        // here exactly as NeoSolver::numeric would and resumed on the device.
        std::vector<int> status(b->count);
        for (int round = 0; round < 1000000; ++round) {
            if ((e = cudaStreamSynchronize(st)) != cudaSuccess ||
                (e = cudaMemcpy(status.data(), b->d_status, sizeof(int) * b->count,
                                cudaMemcpyDeviceToHost)) != cudaSuccess)
                return cuda_fail("nsg_tran_batch_run", e);
            std::vector<int32_t> subset, todo;
            for (int i = 0; i < b->count; ++i)
                if (status[i] == NSG_REORDER || status[i] == 105) todo.push_back(i);
            // The matrices the stopped instances assembled, and their requests.
            const int nt = static_cast<int>(todo.size());
            std::vector<nsg::TranCtl> ctls(nt);
            std::vector<std::vector<double>> mats(nt);
            for (int k = 0; k < nt; ++k) {
                const int i = todo[k];
                const nsg::DcDesc& d = b->descs[i];
                mats[k].resize(d.nnz);
                if ((e = cudaMemcpy(&ctls[k], b->d_ctl + i, sizeof(nsg::TranCtl),
                                    cudaMemcpyDeviceToHost)) != cudaSuccess ||
                    (e = cudaMemcpy(mats[k].data(), b->d_work + d.a_off, sizeof(double) * d.nnz,
                                    cudaMemcpyDeviceToHost)) != cudaSuccess)
                    return cuda_fail("nsg_tran_batch_run", e);
            }
            // Order them on the host threads (instances are independent: a
            // first ordering of a fresh topology, or NeoSolver::numeric on a
            // copy of the current one), then share and place the results.
            // Requests an earlier run answered take its topology.
            b->memo.resize(b->count);
            std::vector<int> from(nt), hit(nt, -1);
            for (int k = 0; k < nt; ++k) {
                const int i = todo[k];
                const nsg::TranCtl& ctl = ctls[k];
                from[k] = ctl.need == 105 ? -1
                                          : (ctl.need_plan == 0 ? b->descs[i].plan
                                                                : b->tdescs[i].tran_plan);
                for (const auto& m : b->memo[i])
                    if (m.need == (ctl.need == 105 ? 105 : 0) && m.from == from[k] &&
                        std::memcmp(&m.diag_gmin, &ctl.need_diag_gmin, sizeof(double)) == 0 &&
                        m.a.size() == mats[k].size() &&
                        std::memcmp(m.a.data(), mats[k].data(), sizeof(double) * m.a.size()) == 0)
                        hit[k] = m.topo;
            }
            std::vector<std::unique_ptr<nsg_topology>> made(nt);
            std::vector<int> rcs(nt, NSG_OK);
            std::atomic<int> next_item{0};
            auto worker = [&]() {
                for (int k; (k = next_item.fetch_add(1)) < nt;) {
                    if (hit[k] >= 0) continue;
                    const int i = todo[k];
                    const nsg::DcDesc& d = b->descs[i];
                    const nsg::TranCtl& ctl = ctls[k];
                    try {
                        if (ctl.need == 105) {
                            rcs[k] = order_topology(d.n, d.nnz, b->col_ptr[i].data(),
                                                    b->row_idx[i].data(), mats[k].data(),
                                                    ctl.need_diag_gmin, made[k], b->solver[i]);
                        } else {
                            made[k] = clone_topology(*b->topos[from[k]]);
                            rcs[k] = numeric_on_engine(*made[k], mats[k].data(), ctl.need_diag_gmin);
                            if (rcs[k] == NSG_OK) rebuild_plan(*made[k]);
                        }
                    } catch (const std::exception&) {
                        rcs[k] = NSG_ERR_INVALID;
                    }
                }
            };
            const int nthreads = std::max(1, std::min<int>(nt, static_cast<int>(std::max(
                                                                 1u, std::thread::hardware_concurrency()))));
            if (nthreads <= 1) {
                worker();
            } else {
                std::vector<std::thread> pool;
                for (int t = 0; t < nthreads; ++t) pool.emplace_back(worker);
                for (auto& th : pool) th.join();
            }
            const size_t ntopos = b->topos.size();
            for (int k = 0; k < nt; ++k) {
                const int i = todo[k];
                int topo = hit[k];
                if (topo < 0) {
                    if (rcs[k] != NSG_OK || !made[k]) continue;  // keeps its status: not ordered
                    topo = intern_topology(b->topos, std::move(made[k]));
                    auto& mi = b->memo[i];
                    if (mi.size() >= 4) mi.erase(mi.begin());
                    mi.push_back({ctls[k].need == 105 ? 105 : 0, from[k], ctls[k].need_diag_gmin,
                                  std::move(mats[k]), topo});
                }
                nsg::DcDesc& d = b->descs[i];
                if (ctls[k].need_plan == 0) d.plan = topo;
                else b->tdescs[i].tran_plan = topo;
                place_lu_workspace(d, b->topos[topo]->plan, b->work_size);
                subset.push_back(i);
                ++b->orderings;
            }
            if (subset.empty()) {
                b->recorded = b->record;
                break;
            }
            if (b->topos.size() != ntopos) {  // new plans to upload
                int rc = refresh_plans(b->topos, &b->d_lu_pool, &b->d_plans, &b->max_col,
                                       &b->max_n);
                if (rc != NSG_OK) return rc;
            }
            if (nsg::tran_smem_bytes(b->max_col, b->max_n) > 200 * 1024)
                return fail(NSG_ERR_INVALID, "nsg_tran_batch_run: an ordered instance is too "
                                             "large for the shared-memory refactor");
            if ((e = grow_workspace(&b->d_work, &b->work_cap, b->work_size)) != cudaSuccess ||
                (e = cudaMemcpy(b->d_descs, b->descs.data(), sizeof(nsg::DcDesc) * b->count,
                                cudaMemcpyHostToDevice)) != cudaSuccess ||
                (e = cudaMemcpy(b->d_tdescs, b->tdescs.data(), sizeof(nsg::TranDesc) * b->count,
                                cudaMemcpyHostToDevice)) != cudaSuccess ||
                (e = cudaMemcpy(b->d_subset, subset.data(), sizeof(int32_t) * subset.size(),
                                cudaMemcpyHostToDevice)) != cudaSuccess ||
                (e = launch(b->d_subset, static_cast<int>(subset.size()))) != cudaSuccess)
                return cuda_fail("nsg_tran_batch_run", e);
        }
        return NSG_OK;
    });
}

int nsg_tran_batch_engines(const nsg_tran_batch* b, int* dc_engine, int* tran_engine) {
    if (!b) return fail(NSG_ERR_INVALID, "nsg_tran_batch_engines: null batch");
    auto kind = [&](int topo) {
        if (topo < 0) return -1;  // not ordered yet
        return b->topos[topo]->plan.kind == nsg::kPlanKindAmdLu ? NSG_SOLVER_AMDLU
                                                                 : NSG_SOLVER_MARKOWITZ;
    };
    for (int i = 0; i < b->count; ++i) {
        if (dc_engine) dc_engine[i] = kind(b->descs[i].plan);
        if (tran_engine) tran_engine[i] = kind(b->tdescs[i].tran_plan);
    }
    return NSG_OK;
}

int nsg_tran_batch_record(nsg_tran_batch* b, int enable) {
    return guarded("nsg_tran_batch_record", [&]() -> int {
        if (!b) return fail(NSG_ERR_INVALID, "nsg_tran_batch_record: null batch");
        b->record = enable != 0;
        if (b->record && !b->d_rec) {
            int64_t nx = 0;
            for (const auto& d : b->descs) nx += d.n;
            cudaError_t e;
            if ((e = upload<nsg::StepRecord>(&b->d_rec, nullptr,
                                             static_cast<size_t>(b->count) * b->opt.max_points)) !=
                    cudaSuccess ||
                (e = upload<double>(&b->d_x0, nullptr, static_cast<size_t>(nx))) != cudaSuccess)
                return cuda_fail("nsg_tran_batch_record", e);
        }
        return NSG_OK;
    });
}

int nsg_tran_batch_set_adjoint_options(nsg_tran_batch* b, double reltol, double vntol,
                                       double abstol, int max_iter) {
    if (!b || !(reltol > 0.0) || !(vntol >= 0.0) || !(abstol >= 0.0) || max_iter < 1)
        return fail(NSG_ERR_INVALID, "nsg_tran_batch_set_adjoint_options: bad arguments");
    b->adj_opt.reltol = reltol;
    b->adj_opt.vntol = vntol;
    b->adj_opt.abstol = abstol;
    b->adj_max_iter = max_iter;
    return NSG_OK;
}

int nsg_tran_batch_params(const nsg_tran_batch* b, long long* offsets, double* params_dc,
                          double* params_tran) {
    if (!b) return fail(NSG_ERR_INVALID, "nsg_tran_batch_params: null batch");
    int64_t total = 0;
    for (int i = 0; i < b->count; ++i) {
        if (offsets) offsets[i] = total;
        total += b->param_count[i];
    }
    if (offsets) offsets[b->count] = total;
    cudaError_t e = cudaSuccess;
    if (params_dc)
        e = cudaMemcpy(params_dc, b->d_params_dc, sizeof(double) * total, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && params_tran)
        e = cudaMemcpy(params_tran, b->d_params_tran, sizeof(double) * total,
                       cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? NSG_OK : cuda_fail("nsg_tran_batch_params", e);
}

int nsg_tran_batch_adjoint(nsg_tran_batch* b, const int* probe, const double* d_targets,
                           double weight, int every, const double* d_params_dc,
                           const double* d_params_tran, double* d_grads, double* d_loss,
                           int* d_status, void* stream) {
    return guarded("nsg_tran_batch_adjoint", [&]() -> int {
        if (!b || !probe || !d_targets || !d_grads || !d_loss || !d_status || every < 1)
            return fail(NSG_ERR_INVALID, "nsg_tran_batch_adjoint: bad arguments");
        if (!b->recorded)
            return fail(NSG_ERR_INVALID, "nsg_tran_batch_adjoint: no recorded run (enable "
                                         "nsg_tran_batch_record before nsg_tran_batch_run)");
        const cudaStream_t st = static_cast<cudaStream_t>(stream);
        std::vector<int> npts(b->count), status(b->count);
        cudaError_t e;
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess ||
            (e = cudaMemcpy(npts.data(), b->d_npoints, sizeof(int) * b->count,
                            cudaMemcpyDeviceToHost)) != cudaSuccess ||
            (e = cudaMemcpy(status.data(), b->d_status, sizeof(int) * b->count,
                            cudaMemcpyDeviceToHost)) != cudaSuccess)
            return cuda_fail("nsg_tran_batch_adjoint", e);
        std::vector<nsg::AdjDesc> ad(b->count);
        int64_t ws = 0;
        for (int i = 0; i < b->count; ++i) {
            const auto& d = b->descs[i];
            const auto& t = b->tdescs[i];
            if (status[i] != 0 || t.tran_plan < 0)
                return fail(NSG_ERR_INVALID, "nsg_tran_batch_adjoint: instance " +
                                                 std::to_string(i) + " has no completed run");
            if (npts[i] >= b->opt.max_points)
                return fail(NSG_ERR_INVALID, "nsg_tran_batch_adjoint: instance " +
                                                 std::to_string(i) +
                                                 " filled max_points; the schedule is incomplete");
            if (!b->adjoint_ok[i])
                return fail(NSG_ERR_INVALID, "nsg_tran_batch_adjoint: instance " +
                                                 std::to_string(i) +
                                                 " has BSIM4v7 devices (not covered)");
            if (probe[i] < 0 || probe[i] >= d.n)
                return fail(NSG_ERR_INVALID, "nsg_tran_batch_adjoint: probe out of range");
            nsg::AdjDesc& a = ad[i];
            a.n_steps = npts[i] - 1;
            a.every = every;
            a.probe = probe[i];
            a.n_ckpt = a.n_steps / every + 1;
            a.rec_off = t.out_off;
            a.x0_off = t.x0_off;
            const int64_t nmos = d.n_mos;
            a.ckpt_len = (2 * d.n + 2 * d.n_states + nsg::kMosRecCount * nmos + 3) & ~int64_t{3};
            a.ws_off = ws;
            ws += a.n_ckpt * a.ckpt_len + (every + 2) * (int64_t{d.n} + d.n_states) +
                  7 * (int64_t{d.n_caps} + d.n_diodes + nsg::kMos1ChargeUnits * nmos) + d.n;
            ws = (ws + 3) & ~int64_t{3};
            // The LU region must hold both the DC and the transient plan.
            const auto& pd = b->topos[d.plan]->plan;
            const auto& pt = b->topos[t.tran_plan]->plan;
            if (pd.nnz_lu > pt.nnz_lu || pd.lrow_ptr[pd.n] > pt.lrow_ptr[pt.n] ||
                pd.urow_ptr[pd.n] > pt.urow_ptr[pt.n]) {
                nsg::TopologyPlan big = pd.nnz_lu >= pt.nnz_lu ? pd : pt;
                big.lrow_ptr[big.n] = std::max(pd.lrow_ptr[pd.n], pt.lrow_ptr[pt.n]);
                big.urow_ptr[big.n] = std::max(pd.urow_ptr[pd.n], pt.urow_ptr[pt.n]);
                place_lu_workspace(b->descs[i], big, b->work_size);
            }
        }
        if ((e = grow_workspace(&b->d_work, &b->work_cap, b->work_size)) != cudaSuccess ||
            (e = cudaMemcpy(b->d_descs, b->descs.data(), sizeof(nsg::DcDesc) * b->count,
                            cudaMemcpyHostToDevice)) != cudaSuccess)
            return cuda_fail("nsg_tran_batch_adjoint", e);
        if (ws > b->adj_ws_cap) {
            cudaFree(b->d_adj_ws);
            b->d_adj_ws = nullptr;
            b->adj_ws_cap = 0;
            if ((e = cudaMalloc(reinterpret_cast<void**>(&b->d_adj_ws), sizeof(double) * ws)) !=
                cudaSuccess)
                return cuda_fail("nsg_tran_batch_adjoint", e);
            b->adj_ws_cap = ws;
        }
        if (!b->d_adescs &&
            (e = upload<nsg::AdjDesc>(&b->d_adescs, nullptr, b->count)) != cudaSuccess)
            return cuda_fail("nsg_tran_batch_adjoint", e);
        int64_t nparam = 0;
        for (auto c : b->param_count) nparam += c;
        if ((e = cudaMemcpy(b->d_adescs, ad.data(), sizeof(nsg::AdjDesc) * b->count,
                            cudaMemcpyHostToDevice)) != cudaSuccess ||
            (e = cudaMemsetAsync(d_grads, 0, sizeof(double) * nparam, st)) != cudaSuccess ||
            (e = nsg::launch_tran_adjoint(
                 b->d_plans, b->d_lu_pool, b->d_descs, b->d_tdescs, b->d_adescs, b->count,
                 b->d_prog, d_params_dc ? d_params_dc : b->d_params_dc,
                 d_params_tran ? d_params_tran : b->d_params_tran, b->d_work, b->d_adj_ws,
                 b->d_rec, b->d_times, b->d_x0, d_targets, weight, d_grads, d_loss, d_status,
                 b->adj_opt, b->adj_max_iter, b->max_col, b->max_n, st)) != cudaSuccess)
            return cuda_fail("nsg_tran_batch_adjoint", e);
        return NSG_OK;
    });
}

int nsg_tran_batch_orderings(const nsg_tran_batch* b, long long* count) {
    if (!b || !count) return fail(NSG_ERR_INVALID, "nsg_tran_batch_orderings: null argument");
    *count = b->orderings;
    return NSG_OK;
}

int nsg_tran_batch_results(const nsg_tran_batch* b, double* times, double* values, int* npoints,
                           int* status, int* stats) {
    if (!b) return fail(NSG_ERR_INVALID, "nsg_tran_batch_results: null batch");
    const size_t nout = static_cast<size_t>(b->count) * b->opt.max_points;
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess && times)
        e = cudaMemcpy(times, b->d_times, sizeof(double) * nout, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && values)
        e = cudaMemcpy(values, b->d_values, sizeof(double) * nout * b->opt.nprobe,
                       cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && npoints)
        e = cudaMemcpy(npoints, b->d_npoints, sizeof(int) * b->count, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && status)
        e = cudaMemcpy(status, b->d_status, sizeof(int) * b->count, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && stats)
        e = cudaMemcpy(stats, b->d_stats, sizeof(int) * 4 * b->count, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? NSG_OK : cuda_fail("nsg_tran_batch_results", e);
}

}  // extern "C"
