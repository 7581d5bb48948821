// C ABI of the batched transient analysis (include/nsgpu.h).
#include "capi_internal.hpp"

#include "host/circuit.hpp"
#include "kernels/tran_device.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <thread>

namespace nsg {
cudaError_t launch_transient(const PlanDesc* plans, const int32_t* lu_pool, const DcDesc* descs,
                             const TranDesc* tdescs, int count, const int32_t* prog,
                             const double* params_dc, const double* params_tran, double* work,
                             const double* bps, const int32_t* probes, double* times,
                             double* values, int32_t* npoints, int32_t* status, int32_t* stats,
                             const TranOptions& o, int max_col, int max_n, cudaStream_t stream);
size_t tran_smem_bytes(int max_col, int max_n);
}  // namespace nsg

using namespace nsg_internal;

struct nsg_tran_batch {
    int count = 0;
    nsg::TranOptions opt{};
    std::vector<std::unique_ptr<nsg_topology>> topos;
    std::vector<long long> param_off;
    std::vector<double> host_params;
    int max_col = 0, max_n = 0;
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
    ~nsg_tran_batch() {
        for (void* p : {static_cast<void*>(d_lu_pool), static_cast<void*>(d_plans),
                        static_cast<void*>(d_prog), static_cast<void*>(d_descs),
                        static_cast<void*>(d_tdescs), static_cast<void*>(d_work),
                        static_cast<void*>(d_params_dc), static_cast<void*>(d_params_tran),
                        static_cast<void*>(d_bps), static_cast<void*>(d_probes),
                        static_cast<void*>(d_times), static_cast<void*>(d_values),
                        static_cast<void*>(d_npoints), static_cast<void*>(d_status),
                        static_cast<void*>(d_stats)})
            cudaFree(p);
    }
};

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
            if (!circuits[i]->c.diodes().empty())
                return fail(NSG_ERR_INVALID,
                            "nsg_tran_batch_create: diodes are not supported in transient yet");
            for (int j = 0; j < nprobe; ++j)
                if (probes[j] < 0 || probes[j] >= circuits[i]->c.num_vars())
                    return fail(NSG_ERR_INVALID, "nsg_tran_batch_create: probe out of range");
        }
        auto b = std::make_unique<nsg_tran_batch>();
        b->count = count;
        if (threads <= 0) threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
        auto& o = b->opt;
        o.nopt = nsg::NewtonOptions{1e-3, 1e-6, 1e-12, 1e-12, 0.0, 100, 0};
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
        // initial dt and the first step's dt, and the two symbolic results
        // (the DC solver and the transient solver each order on their own
        // first matrix, as the reference creates two solvers).
        std::vector<std::vector<double>> ptran(count), bps(count);
        std::vector<double> dt0(count), dt1(count);
        for (int i = 0; i < count; ++i) {
            const auto& c = circuits[i]->c;
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
            // the first loop iteration's clamps (transient.cpp:896-905)
            double d1 = std::max(std::min(dt, o.dt_max), o.dt_min);
            if (!bps[i].empty()) {
                const double bpt = bps[i][0];
                if (d1 > bpt - 1e-18 || d1 > bpt - 0.1 * d1) d1 = bpt;
            }
            if (d1 > tstop) d1 = tstop;
            dt1[i] = d1;
        }
        std::vector<std::unique_ptr<nsg_topology>> ord_dc(count), ord_tr(count);
        std::vector<int> rc_dc(count, NSG_OK), rc_tr(count, NSG_OK);
        std::atomic<int> next{0};
        std::vector<std::thread> pool;
        for (int t = 0; t < std::min(threads, count); ++t)
            pool.emplace_back([&] {
                for (int i; (i = next.fetch_add(1)) < count;) {
                    const auto& c = circuits[i]->c;
                    std::vector<double> a, r;
                    c.initjct_values(a, r, o.nopt.gmin);
                    rc_dc[i] = order_topology(c.num_vars(), c.nnz(), c.col_ptr().data(),
                                              c.row_idx().data(), a.data(), 0.0, ord_dc[i]);
                    c.first_transient_matrix(a, dt1[i], o.nopt.gmin);
                    rc_tr[i] = order_topology(c.num_vars(), c.nnz(), c.col_ptr().data(),
                                              c.row_idx().data(), a.data(), 0.0, ord_tr[i]);
                }
            });
        for (auto& th : pool) th.join();
        for (int i = 0; i < count; ++i)
            if (rc_dc[i] != NSG_OK || rc_tr[i] != NSG_OK)
                return fail(NSG_SINGULAR, "nsg_tran_batch_create: symbolic phase failed for "
                                          "instance " + std::to_string(i));
        auto intern = [&](std::unique_ptr<nsg_topology>& t) -> int {
            for (size_t k = 0; k < b->topos.size(); ++k) {
                const auto& p = b->topos[k]->plan;
                const auto& q = t->plan;
                if (p.n == q.n && p.perm_row == q.perm_row && p.perm_col == q.perm_col &&
                    p.col_ptr == q.col_ptr && p.row_idx == q.row_idx && p.lu_src == q.lu_src)
                    return static_cast<int>(k);
            }
            b->topos.push_back(std::move(t));
            return static_cast<int>(b->topos.size()) - 1;
        };
        std::vector<int> plan_dc(count), plan_tr(count);
        for (int i = 0; i < count; ++i) {
            plan_dc[i] = intern(ord_dc[i]);
            plan_tr[i] = intern(ord_tr[i]);
        }

        std::vector<int32_t> lu_pool, prog;
        std::vector<nsg::PlanDesc> plans;
        for (const auto& t : b->topos) {
            plans.push_back(make_plan_desc(t->plan, lu_pool));
            b->max_col = std::max(b->max_col, t->plan.max_col);
            b->max_n = std::max(b->max_n, t->plan.n);
        }
        std::vector<nsg::DcDesc> descs(count);
        std::vector<nsg::TranDesc> tdescs(count);
        std::vector<double> params_tran, all_bps;
        b->param_off.assign(count + 1, 0);
        int64_t work = 0;
        for (int i = 0; i < count; ++i) {
            const auto& c = circuits[i]->c;
            // workspace sized for the larger of the two LU patterns
            const auto& pd = b->topos[plan_dc[i]]->plan;
            const auto& pt = b->topos[plan_tr[i]]->plan;
            const auto& big = (pd.nnz_lu >= pt.nnz_lu) ? pd : pt;
            nsg::DcDesc& d = descs[i];
            fill_instance(d, c, big, prog, work);
            if (pd.lrow_ptr[pd.n] > big.lrow_ptr[big.n] || pd.urow_ptr[pd.n] > big.urow_ptr[big.n] ||
                pt.lrow_ptr[pt.n] > big.lrow_ptr[big.n] || pt.urow_ptr[pt.n] > big.urow_ptr[big.n]) {
                // row copies sized per plan: give each the larger of the two
                d.lrows_off = work;
                work += (std::max(pd.lrow_ptr[pd.n], pt.lrow_ptr[pt.n]) + 3) & ~3;
                d.urows_off = work;
                work += (std::max(pd.urow_ptr[pd.n], pt.urow_ptr[pt.n]) + 3) & ~3;
            }
            d.index = i;
            d.plan = plan_dc[i];
            d.param_off = b->param_off[i];
            d.sol_off = 0;
            b->param_off[i + 1] = b->param_off[i] + static_cast<int64_t>(c.params().size());
            b->host_params.insert(b->host_params.end(), c.params().begin(), c.params().end());
            params_tran.insert(params_tran.end(), ptran[i].begin(), ptran[i].end());
            nsg::TranDesc& t = tdescs[i];
            t.tran_plan = plan_tr[i];
            t.n_bps = static_cast<int32_t>(bps[i].size());
            t.bp_off = static_cast<int64_t>(all_bps.size());
            all_bps.insert(all_bps.end(), bps[i].begin(), bps[i].end());
            t.out_off = static_cast<int64_t>(i) * max_points;
            t.hist_off = work;
            work += (3 * static_cast<int64_t>(c.num_vars()) + 3) & ~int64_t{3};
            t.dt0 = dt0[i];
        }
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
            (e = upload(&b->d_descs, descs.data(), descs.size())) != cudaSuccess ||
            (e = upload(&b->d_tdescs, tdescs.data(), tdescs.size())) != cudaSuccess ||
            (e = upload<double>(&b->d_work, nullptr, static_cast<size_t>(work))) != cudaSuccess ||
            (e = upload(&b->d_params_dc, b->host_params.data(), b->host_params.size())) != cudaSuccess ||
            (e = upload(&b->d_params_tran, params_tran.data(), params_tran.size())) != cudaSuccess ||
            (e = upload(&b->d_bps, all_bps.data(), all_bps.size())) != cudaSuccess ||
            (e = upload(&b->d_probes, pr.data(), pr.size())) != cudaSuccess ||
            (e = upload<double>(&b->d_times, nullptr, nout)) != cudaSuccess ||
            (e = upload<double>(&b->d_values, nullptr, nout * nprobe)) != cudaSuccess ||
            (e = upload<int32_t>(&b->d_npoints, nullptr, count)) != cudaSuccess ||
            (e = upload<int32_t>(&b->d_status, nullptr, count)) != cudaSuccess ||
            (e = upload<int32_t>(&b->d_stats, nullptr, 4 * static_cast<size_t>(count))) != cudaSuccess)
            return cuda_fail("nsg_tran_batch_create", e);
        *out = b.release();
        return NSG_OK;
    });
}

void nsg_tran_batch_free(nsg_tran_batch* b) { delete b; }

int nsg_tran_batch_run(nsg_tran_batch* b, void* stream) {
    if (!b) return fail(NSG_ERR_INVALID, "nsg_tran_batch_run: null batch");
    cudaError_t e = nsg::launch_transient(
        b->d_plans, b->d_lu_pool, b->d_descs, b->d_tdescs, b->count, b->d_prog, b->d_params_dc,
        b->d_params_tran, b->d_work, b->d_bps, b->d_probes, b->d_times, b->d_values, b->d_npoints,
        b->d_status, b->d_stats, b->opt, b->max_col, b->max_n, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? NSG_OK : cuda_fail("nsg_tran_batch_run", e);
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
