// Batched transient analysis: solve_transient (src/core/transient.cpp:694-1067)
// for one circuit instance per CTA, all instances in one launch, each with its
// own adaptive timestep.  Thread 0 runs the timestep controller
// (TimeStepController, src/core/timestep.cpp) and the accept/reject logic;
// the whole CTA runs each Newton solve, the truncation-error estimate of the
// charge states (ckt_terr, src/devices/ckt_terr.hpp:19-64) and the ringing
// check.  The controller (TranCtl) is kept in shared memory during a launch
// and in global memory between launches: an instance stops whenever one of
// its solvers needs the host (the transient solver's first ordering, or a
// re-ordering after failed pivot re-validation) and resumes where it stopped.
#include "dc_op.cuh"
#include "tran_device.cuh"

#include <cuda_runtime.h>

namespace nsg {

namespace {

// Transient driver constants (src/core/transient.cpp:44-78).
constexpr int kMaxTransientIterations = 500000;
constexpr int kNoRecentBreakpoint = 1000;
constexpr double kNewtonFailureDtFactor = 8.0;
constexpr double kDeviceLteRejectRatio = 0.9;
constexpr double kMaxDtGrowthFactor = 2.0;
constexpr int kRingingMinStepsAfterBp = 5;
constexpr int kLteMinStepCount = 2;

// ckt_terr for the capacitor whose charge is state slot q.
__device__ inline double cap_trunc(const Inst& v, int32_t q, const IntegCtx& c,
                                   const TranOptions& o) {
    const int order = c.order;
    if (order < 1 || c.delta <= 0.0) return 1e30;
    const int ccap = q + 1;
    const double* s0 = v.st[0];
    const double* s1 = v.st[1];
    const double volttol = o.nopt.abstol + o.nopt.reltol * fmax(fabs(s0[ccap]), fabs(s1[ccap]));
    double chargetol = fmax(fabs(s0[q]), fabs(s1[q]));
    chargetol = o.nopt.reltol * fmax(chargetol, o.chgtol) / c.delta;
    const double tol = fmax(volttol, chargetol);
    double diff[4], deltmp[4];
    for (int i = order + 1; i >= 0; --i) diff[i] = v.st[i][q];
    for (int i = 0; i <= order; ++i) deltmp[i] = c.delta_old[i];
    int j = order;
    for (;;) {
        for (int i = 0; i <= j; ++i) diff[i] = (diff[i] - diff[i + 1]) / deltmp[i];
        if (--j < 0) break;
        for (int i = 0; i <= j; ++i) deltmp[i] = deltmp[i + 1] + c.delta_old[i];
    }
    const double gear_coeff[2] = {0.5, 0.2222222222};
    const double trap_coeff[2] = {0.5, 0.08333333333};
    const double factor = (c.method == 1) ? gear_coeff[order - 1] : trap_coeff[order - 1];
    double del = o.trtol * tol / fmax(o.nopt.abstol, factor * fabs(diff[0]));
    if (order == 2) del = sqrt(del);
    return del;
}

// Minimum over the charge states of capacitors, diodes and MOSFETs of their
// proposed timestep (Device::compute_trunc: capacitor.cpp,
// dio_device.cpp:280-290, mos1_device.cpp:352-366,
// bsim4v7_device.cpp:1006-1027), reduced across the CTA.
// std::min semantics: a NaN proposal is ignored.
__device__ inline double min_trunc(const Inst& v, const IntegCtx& c, const TranOptions& o,
                                   double* s_red) {
    double m = 1e30;
    for (int32_t k = threadIdx.x; k < v.n_caps; k += blockDim.x) {
        const double t = cap_trunc(v, v.caps[5 * k + 4], c, o);
        if (t < m) m = t;
    }
    for (int32_t k = threadIdx.x; k < v.n_diodes; k += blockDim.x) {
        const double t = cap_trunc(v, v.diodes[4 * k + 3] + kDsQ, c, o);
        if (t < m) m = t;
    }
    for (int32_t k = threadIdx.x; k < 5 * v.n_mos; k += blockDim.x) {
        const int32_t* mr = v.mos + kMosTabStride * (k / 5);
        const int r = k % 5;
        int q;
        if (mr[6] == kMosFamilyBsim4) {  // qb, qg, qd (BSIM4v7Device::compute_trunc)
            if (r >= 3) continue;
            q = r == 0 ? kB4SQb : r == 1 ? kB4SQg : kB4SQd;
        } else {  // qgs, qgd, qgb, qbd, qbs
            q = r == 0 ? kSQgs : r == 1 ? kSQgd : r == 2 ? kSQgb : r == 3 ? kSQbd : kSQbs;
        }
        const double t = cap_trunc(v, mr[5] + q, c, o);
        if (t < m) m = t;
    }
    for (int off = 16; off > 0; off >>= 1) {
        const double other = __shfl_xor_sync(0xffffffffu, m, off);
        if (other < m) m = other;
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = m;
    __syncthreads();
    double r = 1e30;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
        if (s_red[w] < r) r = s_red[w];
    __syncthreads();
    return r;
}

__device__ inline void store_point(const TranDesc& td, const TranOptions& o,
                                   const int32_t* probes, double* times, double* values,
                                   int p, double t, const double* sol) {
    if (p >= o.max_points) return;
    for (int32_t j = threadIdx.x; j < o.nprobe; j += blockDim.x)
        values[(td.out_off + p) * o.nprobe + j] = sol[probes[j]];
    if (threadIdx.x == 0) times[td.out_off + p] = t;
}

// The step's clamps (transient.cpp:890-905) and fill_integrator_context
// (transient.cpp:398-448).  Thread 0.  Returns false when the loop ends.
__device__ inline bool prepare_step(TranCtl& k, const TranDesc& td, const double* bp,
                                    const TranOptions& o) {
    if (!(k.time < o.tstop - 1e-18)) return false;
    if (++k.total_iterations > kMaxTransientIterations) {
        k.status = kTranTooManySteps;
        return false;
    }
    double dt = k.dt;
    dt = fmin(dt, o.dt_max);
    dt = fmax(dt, o.dt_min);
    const double unclamped = dt;
    if (k.bp_head < td.n_bps) {  // clamp_to_breakpoint
        const double b = bp[k.bp_head];
        const double t_next = k.time + dt;
        if (t_next > b - 1e-18 || t_next > b - 0.1 * dt) dt = b - k.time;
    }
    if (dt < unclamped - 1e-18) k.saved_delta = unclamped;
    if (k.time + dt > o.tstop) dt = o.tstop - k.time;  // clamp_to_end
    if (dt < 1e-20) return false;
    k.dt = dt;
    IntegCtx& c = k.ctx;
    const bool first = (k.step_count == 0);
    c.order = k.order;
    c.delta = dt;
    c.time = k.time + dt;
    c.delta_old[0] = dt;
    c.delta_old[1] = first ? dt : k.prev_dt;
    c.delta_old[2] = k.prev_prev_dt;
    k.step_mode = kModeTran | (first ? kModeInitTran : kModeInitPred);
    c.mode = k.step_mode;
    if (k.order == 1) {
        c.ag[0] = 1.0 / dt;
        c.ag[1] = -1.0 / dt;
        c.ag[2] = 0.0;
        c.xmu_ratio = 0.0;
    } else if (c.method != 1) {
        const double one_minus_xmu = 1.0 - o.xmu;
        c.ag[0] = 1.0 / (dt * one_minus_xmu);
        c.ag[1] = -1.0 / (dt * one_minus_xmu);
        c.ag[2] = 0.0;
        c.xmu_ratio = o.xmu / one_minus_xmu;
    } else {
        const double h_old = k.prev_dt;
        if (h_old > 0.0) {
            const double sum = dt + h_old;
            c.ag[0] = (2.0 * dt + h_old) / (dt * sum);
            c.ag[1] = -(dt + h_old) / (dt * h_old);
            c.ag[2] = dt / (h_old * sum);
        } else {
            c.ag[0] = 1.0 / dt;
            c.ag[1] = -1.0 / dt;
            c.ag[2] = 0.0;
        }
        c.xmu_ratio = 0.0;
    }
    return true;
}

// Copy the stage back, then (thread 0) write the controller back and report
// the instance.
__device__ inline void finish(const DcDesc& d, double* work, double* stage, TranCtl* g,
                              const TranCtl& k, const TranOptions& o, int32_t* npoints,
                              int32_t* status, int32_t* stats, int32_t code) {
    stage_copy(d, work, stage, false);
    if (threadIdx.x != 0) return;
    *g = k;
    status[d.index] = code;
    npoints[d.index] = k.points < o.max_points ? k.points : o.max_points;
    stats[4 * d.index] = k.step_count;
    stats[4 * d.index + 1] = k.rejected;
    stats[4 * d.index + 2] = k.newton_iters;
    stats[4 * d.index + 3] = k.dc.code;
}

}  // namespace

// One CTA of kThreads threads per instance, kBlocks CTAs per SM (registers
// capped at 65536 / (kThreads * kBlocks)).  subset (optional): descriptor
// positions to run.
template <int kThreads, int kBlocks>
__global__ void __launch_bounds__(kThreads, kBlocks)
transient_kernel(const PlanDesc* __restrict__ plans, const int32_t* __restrict__ lu_pool,
                 const DcDesc* __restrict__ descs, const TranDesc* __restrict__ tdescs,
                 const int32_t* __restrict__ subset, const int32_t* __restrict__ prog,
                 const double* __restrict__ params_dc, const double* __restrict__ params_tran,
                 double* __restrict__ work, const double* __restrict__ bps,
                 const int32_t* __restrict__ probes, double* __restrict__ times,
                 double* __restrict__ values, int32_t* __restrict__ npoints,
                 int32_t* __restrict__ status, int32_t* __restrict__ stats,
                 TranCtl* __restrict__ ctls, TranOptions o_in, int colbuf, int scratch_doubles,
                 int stage_doubles, StepRecord* __restrict__ rec_steps,
                 double* __restrict__ rec_x0, int plan_words) {
    extern __shared__ double smem[];
    const int pos = subset ? subset[blockIdx.x] : blockIdx.x;
    const DcDesc d = descs[pos];
    const TranDesc td = tdescs[pos];
    TranCtl* const g = ctls + d.index;
    __shared__ TranCtl k;
    __shared__ double s_red[kFlowWarps];
    __shared__ int32_t s_flag;
    double* stage = (d.stage_len <= stage_doubles) ? smem + scratch_doubles : nullptr;
    stage_copy(d, work, stage, true);
    // The instance's views, once per CTA in shared memory (a per-thread copy
    // would sit in every thread's stack frame, far beyond L1).
    __shared__ Inst s_v;
    if (threadIdx.x == 0) s_v = make_inst(d, prog, params_dc, work, stage);
    Inst& v = s_v;
    double* hist = ws_at(d, work, stage, td.hist_off);  // three history vectors (ring)
    const double* bp = bps + td.bp_off;
    constexpr int kFirst = kModeTranOp | kModeInitJct, kCont = kModeTranOp | kModeInitFloat;

    // Options by reference from shared memory, not from a per-thread copy.
    __shared__ TranOptions s_o;
    if (threadIdx.x == 0) {
        k = *g;
        s_o = o_in;
    }
    __syncthreads();
    const TranOptions& o = s_o;
    if (k.phase == kTrInit) {
        for (int32_t i = threadIdx.x; i < kMosRecCount * v.n_mos; i += blockDim.x) v.mrec[i] = 0.0;
        for (int32_t i = threadIdx.x; i < 4 * d.n_states; i += blockDim.x) v.st[0][i] = 0.0;
        for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) v.x[i] = 0.0;
        if (threadIdx.x == 0) {
            dc_op_start(&k.dc, kFirst, o.nopt.first_aid);
            k.ctx = IntegCtx{};
            k.ctx.order = 1;
            k.ctx.method = o.use_gear;
            for (int q = 0; q < 4; ++q) k.stperm[q] = q;
            k.dc_solver.factored = 0;
            k.tr_solver.factored = 0;
            k.status = kTranOk;
            k.phase = kTrDc;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double* base = ws_at(d, work, stage, d.state_off);
        for (int q = 0; q < 4; ++q) v.st[q] = base + static_cast<int64_t>(k.stperm[q]) * d.n_states;
    }
    __syncthreads();

    // Small instances read their plan from shared memory (the DC plan now,
    // the transient plan for the timestep loop).
    int32_t* plan_sm =
        plan_words > 0 ? reinterpret_cast<int32_t*>(smem + scratch_doubles + stage_doubles) : nullptr;
    __shared__ PlanDesc s_pd;

    // ---- 1. DC operating point (compute_dc_operating_point, transient.cpp:145-205)
    if (k.phase == kTrDc) {
        const int32_t* dpool = stage_plan(plans[d.plan], lu_pool, plan_sm, plan_words, &s_pd);
        const int32_t code = dc_operating_point(v, d.n_states, s_pd, dpool, &k.ctx,
                                                &k.dc_solver, &k.dc, o.nopt, kFirst, kCont, false,
                                                work + d.dcsave_off, smem, colbuf, scratch_doubles);
        if (code == kStatusReorder) {
            if (threadIdx.x == 0) {
                k.need = kStatusReorder;
                k.need_plan = 0;
                k.need_diag_gmin = k.dc.numeric_diag_gmin;
            }
            finish(d, work, stage, g, k, o, npoints, status, stats, kStatusReorder);
            return;
        }
        if (code != kDcConverged) {
            if (threadIdx.x == 0) k.phase = kTrDone;
            finish(d, work, stage, g, k, o, npoints, status, stats,
                   code == kStatusTimeout ? code : kTranDcFailed);
            return;
        }
        // ---- 2. seed the state history from the operating point; t = 0 point
        for (int32_t i = threadIdx.x; i < d.n_states; i += blockDim.x)
            v.st[1][i] = v.st[2][i] = v.st[3][i] = v.st[0][i];
        for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x)
            hist[i] = hist[v.n + i] = hist[2 * v.n + i] = v.x[i];
        store_point(td, o, probes, times, values, 0, 0.0, v.x);
        if (rec_x0)
            for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) rec_x0[td.x0_off + i] = v.x[i];
        if (threadIdx.x == 0) {
            k.points = 1;
            k.hist[0] = 0;
            k.hist[1] = 1;
            k.hist[2] = 2;
            k.newton_iters = k.dc.total;
            k.order = 1;
            k.steps_after_bp = kNoRecentBreakpoint;
            k.dt = td.dt0;
            k.saved_delta = td.dt0;
            k.prev_prev_dt = td.dt0;
            k.proposed_dt = o.tstep;
            k.ctx.method = o.use_gear;
            k.phase = kTrPrepare;
        }
        __syncthreads();
    }
    __syncthreads();
    if (threadIdx.x == 0) v.par = params_tran + d.param_off;  // PULSE defaults resolved
    __syncthreads();
    load_constants(v, o.nopt.gmin);

    // ---- 3. the adaptive timestep loop (transient.cpp:873-1052)
    const bool host_first = td.tran_plan < 0;
    const int32_t* tpool =
        stage_plan(plans[host_first ? d.plan : td.tran_plan], lu_pool, plan_sm, plan_words, &s_pd);
    const PlanDesc& tpd = s_pd;
    for (;;) {
        __syncthreads();
        if (k.phase == kTrPrepare) {
            if (threadIdx.x == 0) k.phase = prepare_step(k, td, bp, o) ? kTrStep : kTrDone;
            __syncthreads();
        }
        if (k.phase == kTrDone) break;

        // Newton at the new timepoint (itl4 iterations), possibly resumed.
        const bool resume = k.nr_active != 0;
        const int nr_iter = k.nr_iter, nr_devconv = k.nr_devconv, step_mode = k.step_mode;
        __syncthreads();
        if (threadIdx.x == 0 && resume) k.ctx.mode = k.nr_mode;
        __syncthreads();
        const NewtonOutcome r = newton(v, tpd, tpool, &k.ctx, o.nopt, o.itl4, &k.tr_solver, smem,
                                       colbuf, resume ? nr_iter : -1, step_mode,
                                       resume ? nr_devconv : 1, host_first, scratch_doubles);
        if (r.code == kStatusReorder || r.code == kStatusNeedOrder) {
            if (threadIdx.x == 0) {
                k.nr_active = 1;
                k.nr_iter = r.fail_iter;
                k.nr_mode = r.fail_mode;
                k.nr_devconv = r.fail_dev_conv;
                k.need = r.code;
                k.need_plan = 1;
                k.need_diag_gmin = o.nopt.diag_gmin;
            }
            finish(d, work, stage, g, k, o, npoints, status, stats, r.code);
            return;
        }
        if (threadIdx.x == 0) k.nr_active = 0;
        if (r.code == kStatusTimeout) {
            if (threadIdx.x == 0) k.status = r.code;
            break;
        }
        double* sol_prev = hist + k.hist[0] * v.n;
        double* sol_prev3 = hist + k.hist[2] * v.n;
        if (r.code != kDcConverged) {
            // Newton failure: dt /= 8, backward Euler, restore (transient.cpp:916-945).
            __syncthreads();
            if (threadIdx.x == 0) {
                k.dt /= kNewtonFailureDtFactor;
                k.order = 1;
                k.order_cooldown = 5;
                if (k.dt < o.dt_min) {
                    if (!k.tried_delmin) {
                        k.dt = o.dt_min;
                        k.tried_delmin = 1;
                    } else {
                        k.status = kTranNewtonFailed;
                    }
                }
                k.phase = kTrPrepare;
            }
            for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) v.x[i] = sol_prev[i];
            __syncthreads();
            if (k.status != kTranOk) break;
            continue;
        }
        if (threadIdx.x == 0) k.newton_iters += r.iters;

        // Device LTE (evaluate_lte, transient.cpp:469-513).
        double device_dt = 1e30;
        if (k.step_count >= kLteMinStepCount) device_dt = min_trunc(v, k.ctx, o, s_red);
        if (threadIdx.x == 0) {
            bool accepted = true;
            if (k.step_count >= kLteMinStepCount) {
                device_dt = fmin(kMaxDtGrowthFactor * k.dt, device_dt);
                if (device_dt < k.dt * kDeviceLteRejectRatio && k.dt > o.dt_min * 1.01) {
                    accepted = false;
                    k.rejected++;
                }
            }
            k.device_dt = device_dt;
            s_flag = accepted ? 0 : 1;
            if (!accepted) {
                double proposed = k.proposed_dt;
                if (device_dt < proposed) proposed = device_dt;
                k.dt = fmax(proposed, o.dt_min);
                k.phase = kTrPrepare;
            }
        }
        __syncthreads();
        if (s_flag) {
            for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) v.x[i] = sol_prev[i];
            continue;
        }

        // Accept (transient.cpp:966-1051).
        if (threadIdx.x == 0) {
            if (rec_steps && k.points < o.max_points) {
                StepRecord& r = rec_steps[td.out_off + k.points];
                for (int q = 0; q < 3; ++q) r.ag[q] = k.ctx.ag[q];
                r.xmu_ratio = k.ctx.xmu_ratio;
                r.order = k.ctx.order;
                r.method = k.ctx.method;
            }
            const double dt = k.dt;
            k.prev_prev_dt = k.prev_dt;
            k.prev_dt = dt;
            k.time += dt;  // advance: consume breakpoints up to the new time
            k.crossed_src_bp = 0;
            while (k.bp_head < td.n_bps && bp[k.bp_head] <= k.time + 1e-18) {
                k.bp_head++;
                k.crossed_src_bp = 1;
            }
            k.step_count++;
            k.tried_delmin = 0;
            if (k.steps_after_bp < kNoRecentBreakpoint) ++k.steps_after_bp;
            if (k.crossed_src_bp && k.step_count > 2) {
                k.steps_after_bp = 0;
                k.order = 1;
                const double gap = (k.bp_head < td.n_bps) ? bp[k.bp_head] - k.time : o.tstop - k.time;
                k.dt = fmin(k.dt, o.restart_scale * fmin(k.saved_delta, gap));
                k.dt = fmax(k.dt, o.dt_min * 2.0);
            }
            if (k.order_cooldown > 0) --k.order_cooldown;
            k.ctx.order = 2;  // for the promotion test below
        }
        __syncthreads();
        const bool try_promote = (k.order == 1 && k.step_count >= 2 && k.order_cooldown == 0);
        double dt2 = 1e30;
        if (try_promote) dt2 = min_trunc(v, k.ctx, o, s_red);
        __syncthreads();
        if (threadIdx.x == 0) {
            if (try_promote && dt2 > 1.05 * k.dt) k.order = 2;
            k.ctx.order = k.order;
        }
        // rotate_state (circuit.cpp:328): state3 <- state2 <- state1, state1 = state0
        if (threadIdx.x == 0) {
            double* t3 = v.st[3];
            v.st[3] = v.st[2];
            v.st[2] = v.st[1];
            v.st[1] = t3;
        }
        __syncthreads();
        for (int32_t i = threadIdx.x; i < d.n_states; i += blockDim.x) v.st[1][i] = v.st[0][i];
        store_point(td, o, probes, times, values, k.points, k.time, v.x);
        for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) sol_prev3[i] = v.x[i];
        __syncthreads();
        if (threadIdx.x == 0) {
            const int32_t p3 = k.stperm[3];
            k.stperm[3] = k.stperm[2];
            k.stperm[2] = k.stperm[1];
            k.stperm[1] = p3;
            k.points++;
            const int h3 = k.hist[2];
            k.hist[2] = k.hist[1];
            k.hist[1] = k.hist[0];
            k.hist[0] = h3;
            s_flag = 0;
        }
        __syncthreads();
        // Ringing detection (detect_and_handle_ringing, transient.cpp:580-606).
        const bool check = (k.step_count >= 3 && !o.use_gear && k.steps_after_bp >= kRingingMinStepsAfterBp);
        if (check) {
            const double* s = v.x;
            const double* p1 = hist + k.hist[0] * v.n;
            const double* p2 = hist + k.hist[1] * v.n;
            const double* p3 = hist + k.hist[2] * v.n;
            for (int32_t i = threadIdx.x; i < v.num_nodes; i += blockDim.x) {
                const double d2c = s[i] - 2.0 * p1[i] + p2[i];
                const double d2p = p1[i] - 2.0 * p2[i] + p3[i];
                const double tol = o.nopt.reltol * fabs(s[i]) + o.nopt.vntol;
                if (d2c * d2p < 0.0 && fabs(d2c) > tol && fabs(d2p) > tol) {
                    const double d1c = s[i] - p1[i];
                    const double d1p = p1[i] - p2[i];
                    double d1max = fmax(fabs(d1c), fabs(d1p));
                    if (d1max < 1e-30) d1max = 1e-30;
                    if (fmax(fabs(d2c), fabs(d2p)) / d1max > 0.5) s_flag = 1;
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            if (check) {
                k.ringing = (s_flag != 0);
                if (k.ringing) k.ringing_cooldown = 3;
                else if (k.ringing_cooldown > 0) --k.ringing_cooldown;  // tick_cooldown
                k.ctx.method = (k.ringing || k.ringing_cooldown > 0) ? 1 : 0;
            }
            if (k.step_count >= kLteMinStepCount) {
                double proposed = k.device_dt;
                proposed = fmin(proposed, kMaxDtGrowthFactor * k.dt);
                k.dt = fmax(proposed, o.dt_min);
            }
            k.phase = kTrPrepare;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) k.phase = kTrDone;
    finish(d, work, stage, g, k, o, npoints, status, stats, k.status);
}

size_t tran_smem_bytes(int max_col, int max_n) {
    const int colbuf = (max_col + 31) & ~31;
    const size_t a = flow_smem_bytes(colbuf, max_n);
    const size_t b = flow_solve_smem_bytes(max_n);
    return a > b ? a : b;
}

namespace {

template <int kThreads, int kBlocks>
cudaError_t configure_transient() {
    static bool configured = false;
    if (configured) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(transient_kernel<kThreads, kBlocks>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e == cudaSuccess) configured = true;
    return e;
}

int sm_count() {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 1;
    }
    return sms;
}

}  // namespace

// Launch shapes.  Latency of one instance is the cost for a few hundred
// instances: one 512-thread CTA per instance, two per SM, each staging its
// plan and workspace in shared memory.  When every instance takes the
// shared-memory LU path (n <= 128) and the batch is larger than those two
// CTAs per SM can hold at once, throughput is the cost: CTAs of 128 or 256
// threads (as many as the instances' largest device family needs for one
// pass of the device loads), eight or four per SM, with the LU and the plan
// in shared memory and the workspace staged only where it fits.  (Two
// 256-thread CTAs per SM at 128 registers spill less in the BSIM4v7 loads
// but ran 20 % slower than four at 64 on the ring + NAND Monte Carlo.)
// sh.force_threads / force_blocks (0: automatic) override the choice.
cudaError_t launch_transient(const PlanDesc* plans, const int32_t* lu_pool, const DcDesc* descs,
                             const TranDesc* tdescs, const int32_t* subset, int count,
                             const int32_t* prog, const double* params_dc,
                             const double* params_tran, double* work, const double* bps,
                             const int32_t* probes, double* times, double* values,
                             int32_t* npoints, int32_t* status, int32_t* stats, TranCtl* ctls,
                             const TranOptions& o, const TranShape& sh,
                             StepRecord* rec_steps, double* rec_x0, cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    const int colbuf = (sh.max_col + 31) & ~31;
    int threads = kFlowThreads, blocks = 2;
    if (sh.max_n <= 128 && count > 2 * sm_count()) {
        threads = sh.max_devices <= 128 ? 128 : (sh.max_devices <= 256 ? 256 : kFlowThreads);
        blocks = threads == 128 ? 8 : (threads == 256 ? 4 : 2);
    }
    if (sh.force_threads > 0) {
        threads = sh.force_threads;
        blocks = sh.force_blocks > 0 ? sh.force_blocks : 1024 / threads;
    }
    const bool small_shape = threads != kFlowThreads;
    if (small_shape && sh.max_n > 128) return cudaErrorInvalidValue;
    size_t scratch, plan, stage;
    if (!small_shape) {
        scratch = (tran_smem_bytes(sh.max_col, sh.max_n) + 15) & ~size_t{15};
        plan = (sh.max_n <= 128) ? kPlanStageBytes : 0;
        stage = stage_bytes_for(scratch + plan, sh.max_stage);
    } else {
        // Per-CTA share of the SM's 228 KB, less the CTA's static shared
        // memory and the 1 KB the runtime reserves per CTA.
        const size_t budget = (228 * 1024) / static_cast<size_t>(blocks) - 3 * 1024;
        scratch = (sizeof(double) * static_cast<size_t>(sh.max_small_lu) + 15) & ~size_t{15};
        plan = (sh.max_plan_words * 4 <= static_cast<int64_t>(kPlanStageBytes))
                   ? ((static_cast<size_t>(sh.max_plan_words) * 4 + 15) & ~size_t{15})
                   : 0;
        if (scratch + plan > budget) plan = 0;
        const size_t want = static_cast<size_t>(sh.max_stage) * sizeof(double);
        stage = (scratch + plan + want <= budget) ? want : 0;
    }
    const size_t smem = scratch + stage + plan;
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    const int scratch_d = static_cast<int>(scratch / sizeof(double));
    const int stage_d = static_cast<int>(stage / sizeof(double));
    const int plan_w = static_cast<int>(plan / sizeof(int32_t));
    cudaError_t e;
#define NSG_LAUNCH_TRAN(T, B)                                                                  \
    if ((e = configure_transient<T, B>()) != cudaSuccess) return e;                            \
    transient_kernel<T, B><<<count, T, smem, stream>>>(                                        \
        plans, lu_pool, descs, tdescs, subset, prog, params_dc, params_tran, work, bps, probes, \
        times, values, npoints, status, stats, ctls, o, colbuf, scratch_d, stage_d, rec_steps,  \
        rec_x0, plan_w);
    if (threads == 128 && blocks == 8) {
        NSG_LAUNCH_TRAN(128, 8)
    } else if (threads == 256 && blocks == 4) {
        NSG_LAUNCH_TRAN(256, 4)
    } else if (threads == kFlowThreads && blocks == 2) {
        NSG_LAUNCH_TRAN(kFlowThreads, 2)
    } else {
        return cudaErrorInvalidValue;
    }
#undef NSG_LAUNCH_TRAN
    return cudaGetLastError();
}

}  // namespace nsg
