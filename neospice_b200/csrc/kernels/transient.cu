// Batched transient analysis: solve_transient (src/core/transient.cpp:694-1067)
// for one circuit instance per CTA, all instances in one launch, each with its
// own adaptive timestep.  Thread 0 runs the timestep controller
// (TimeStepController, src/core/timestep.cpp) and the accept/reject logic;
// the whole CTA runs each Newton solve, the capacitor truncation-error
// estimate (ckt_terr, src/devices/ckt_terr.hpp:19-64) and the ringing check.
#include "newton_common.cuh"
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

// Minimum over capacitors of their proposed timestep (device compute_trunc),
// reduced across the CTA.  std::min semantics: a NaN proposal is ignored.
__device__ inline double min_trunc(const Inst& v, const IntegCtx& c, const TranOptions& o,
                                   double* s_red) {
    double m = 1e30;
    for (int32_t k = threadIdx.x; k < v.n_caps; k += blockDim.x) {
        const double t = cap_trunc(v, v.caps[5 * k + 4], c, o);
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

// Controller state of one instance (thread 0 writes, all read after a barrier).
struct Ctrl {
    double time, dt, prev_dt, prev_prev_dt, saved_delta, proposed_dt, device_dt;
    int order, step_count, steps_after_bp, order_cooldown, ringing_cooldown, rejected;
    int total_iterations, newton_iters, bp_head, points;
    bool tried_delmin, crossed_src_bp, ringing;
    int32_t status;   // kTran* when finished
    int phase;        // what the CTA does next
};

enum : int { kPhaseNewton = 0, kPhaseDone = 1 };

__device__ inline void store_point(const Inst& v, const TranDesc& td, const TranOptions& o,
                                   const int32_t* probes, double* times, double* values,
                                   Ctrl* k, double t, const double* sol) {
    const int p = k->points;
    if (p >= o.max_points) return;
    for (int32_t j = threadIdx.x; j < o.nprobe; j += blockDim.x)
        values[(td.out_off + p) * o.nprobe + j] = sol[probes[j]];
    if (threadIdx.x == 0) times[td.out_off + p] = t;
}

}  // namespace

__global__ void __launch_bounds__(kFlowThreads, 2)
transient_kernel(const PlanDesc* __restrict__ plans, const int32_t* __restrict__ lu_pool,
                 const DcDesc* __restrict__ descs, const TranDesc* __restrict__ tdescs,
                 const int32_t* __restrict__ prog, const double* __restrict__ params_dc,
                 const double* __restrict__ params_tran, double* __restrict__ work,
                 const double* __restrict__ bps, const int32_t* __restrict__ probes,
                 double* __restrict__ times, double* __restrict__ values,
                 int32_t* __restrict__ npoints, int32_t* __restrict__ status,
                 int32_t* __restrict__ stats, TranOptions o, int colbuf) {
    extern __shared__ double smem[];
    const DcDesc d = descs[blockIdx.x];
    const TranDesc td = tdescs[blockIdx.x];
    Inst v = make_inst(d, prog, params_dc, work);
    double* hist = work + td.hist_off;  // sol_prev, sol_prev2, sol_prev3
    const double* bp = bps + td.bp_off;
    __shared__ IntegCtx ctx;
    __shared__ SolverState dc_solver, tr_solver;
    __shared__ Ctrl k;
    __shared__ double s_red[kFlowWarps];
    __shared__ int32_t s_ring;
    __shared__ int s_hist[3];

    // ---- 1. DC operating point (MODETRANOP | MODEINITJCT, transient.cpp:145-205)
    load_constants(v, o.nopt.gmin);
    for (int32_t i = threadIdx.x; i < 3 * v.n_diodes; i += blockDim.x) v.dstate[i] = 0.0;
    for (int32_t i = threadIdx.x; i < 4 * d.n_states; i += blockDim.x) v.st[0][i] = 0.0;
    for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) v.x[i] = 0.0;
    if (threadIdx.x == 0) {
        ctx = IntegCtx{};
        ctx.mode = kModeTranOp | kModeInitJct;
        ctx.order = 1;
        ctx.method = o.use_gear;
        ctx.time = 0.0;
        dc_solver.factored = false;
        tr_solver.factored = false;
        k = Ctrl{};
    }
    __syncthreads();
    NewtonOutcome r = newton(v, plans[d.plan], lu_pool, &ctx, o.nopt, o.nopt.max_iter, &dc_solver,
                             smem, colbuf);
    if (r.code != kDcConverged) {
        if (threadIdx.x == 0) {
            status[d.index] = kTranDcFailed;
            npoints[d.index] = 0;
            stats[4 * d.index] = 0;
            stats[4 * d.index + 1] = 0;
            stats[4 * d.index + 2] = r.iters;
            stats[4 * d.index + 3] = r.code;
        }
        return;
    }

    // ---- 2. seed the state history from the operating point; t = 0 point
    for (int32_t i = threadIdx.x; i < d.n_states; i += blockDim.x)
        v.st[1][i] = v.st[2][i] = v.st[3][i] = v.st[0][i];
    for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x)
        hist[i] = hist[v.n + i] = hist[2 * v.n + i] = v.x[i];
    v.par = params_tran + d.param_off;  // PULSE defaults resolved for the transient
    load_constants(v, o.nopt.gmin);
    if (threadIdx.x == 0) {
        s_hist[0] = 0;
        s_hist[1] = 1;
        s_hist[2] = 2;
        k.newton_iters = r.iters;
        k.order = 1;
        k.steps_after_bp = kNoRecentBreakpoint;
        k.dt = td.dt0;
        k.saved_delta = td.dt0;
        k.prev_prev_dt = td.dt0;
        k.proposed_dt = o.tstep;
        k.phase = kPhaseNewton;
        k.status = kTranOk;
        ctx.method = o.use_gear;
    }
    __syncthreads();
    store_point(v, td, o, probes, times, values, &k, 0.0, v.x);
    if (threadIdx.x == 0) k.points = 1;
    __syncthreads();

    // ---- 3. the adaptive timestep loop (transient.cpp:873-1052)
    for (;;) {
        // Controller, step preparation.
        if (threadIdx.x == 0) {
            k.phase = kPhaseNewton;
            if (!(k.time < o.tstop - 1e-18)) {
                k.phase = kPhaseDone;
            } else if (++k.total_iterations > kMaxTransientIterations) {
                k.status = kTranTooManySteps;
                k.phase = kPhaseDone;
            } else {
                double dt = k.dt;
                dt = fmin(dt, o.dt_max);
                dt = fmax(dt, o.dt_min);
                const double unclamped = dt;
                // clamp_to_breakpoint
                if (k.bp_head < td.n_bps) {
                    const double b = bp[k.bp_head];
                    const double t_next = k.time + dt;
                    if (t_next > b - 1e-18 || t_next > b - 0.1 * dt) dt = b - k.time;
                }
                if (dt < unclamped - 1e-18) k.saved_delta = unclamped;
                if (k.time + dt > o.tstop) dt = o.tstop - k.time;  // clamp_to_end
                if (dt < 1e-20) {
                    k.phase = kPhaseDone;
                } else {
                    k.dt = dt;
                    // fill_integrator_context (transient.cpp:398-448)
                    const bool first = (k.step_count == 0);
                    ctx.order = k.order;
                    ctx.delta = dt;
                    ctx.time = k.time + dt;
                    ctx.delta_old[0] = dt;
                    ctx.delta_old[1] = first ? dt : k.prev_dt;
                    ctx.delta_old[2] = k.prev_prev_dt;
                    ctx.mode = kModeTran | (first ? kModeInitTran : kModeInitPred);
                    if (k.order == 1) {
                        ctx.ag[0] = 1.0 / dt;
                        ctx.ag[1] = -1.0 / dt;
                        ctx.ag[2] = 0.0;
                        ctx.xmu_ratio = 0.0;
                    } else if (ctx.method != 1) {
                        const double one_minus_xmu = 1.0 - o.xmu;
                        ctx.ag[0] = 1.0 / (dt * one_minus_xmu);
                        ctx.ag[1] = -1.0 / (dt * one_minus_xmu);
                        ctx.ag[2] = 0.0;
                        ctx.xmu_ratio = o.xmu / one_minus_xmu;
                    } else {
                        const double h_old = k.prev_dt;
                        if (h_old > 0.0) {
                            const double sum = dt + h_old;
                            ctx.ag[0] = (2.0 * dt + h_old) / (dt * sum);
                            ctx.ag[1] = -(dt + h_old) / (dt * h_old);
                            ctx.ag[2] = dt / (h_old * sum);
                        } else {
                            ctx.ag[0] = 1.0 / dt;
                            ctx.ag[1] = -1.0 / dt;
                            ctx.ag[2] = 0.0;
                        }
                        ctx.xmu_ratio = 0.0;
                    }
                }
            }
        }
        __syncthreads();
        if (k.phase == kPhaseDone) break;

        // Newton at the new timepoint (itl4 iterations).
        r = newton(v, plans[td.tran_plan], lu_pool, &ctx, o.nopt, o.itl4, &tr_solver, smem, colbuf);
        if (r.code == kStatusTimeout || r.code == kStatusReorder) {
            if (threadIdx.x == 0) k.status = r.code;
            __syncthreads();
            break;
        }
        double* sol_prev = hist + s_hist[0] * v.n;
        double* sol_prev3 = hist + s_hist[2] * v.n;
        if (r.code != kDcConverged) {
            // Newton failure: dt /= 8, backward Euler, restore (transient.cpp:916-945).
            if (threadIdx.x == 0) {
                k.dt /= kNewtonFailureDtFactor;
                k.order = 1;
                k.order_cooldown = 5;
                if (k.dt < o.dt_min) {
                    if (!k.tried_delmin) {
                        k.dt = o.dt_min;
                        k.tried_delmin = true;
                    } else {
                        k.status = kTranNewtonFailed;
                    }
                }
            }
            __syncthreads();
            for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) v.x[i] = sol_prev[i];
            __syncthreads();
            if (k.status != kTranOk) break;
            continue;
        }
        if (threadIdx.x == 0) k.newton_iters += r.iters;

        // Device LTE (evaluate_lte, transient.cpp:469-513).
        double device_dt = 1e30;
        if (k.step_count >= kLteMinStepCount) device_dt = min_trunc(v, ctx, o, s_red);
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
            k.phase = accepted ? kPhaseNewton : -1;
            if (!accepted) {
                double proposed = k.proposed_dt;
                if (device_dt < proposed) proposed = device_dt;
                k.dt = fmax(proposed, o.dt_min);
            }
        }
        __syncthreads();
        if (k.phase == -1) {
            for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) v.x[i] = sol_prev[i];
            __syncthreads();
            continue;
        }

        // Accept (transient.cpp:966-1051).
        if (threadIdx.x == 0) {
            const double dt = k.dt;
            k.prev_prev_dt = k.prev_dt;
            k.prev_dt = dt;
            // advance: consume breakpoints up to the new time
            k.time += dt;
            k.crossed_src_bp = false;
            while (k.bp_head < td.n_bps && bp[k.bp_head] <= k.time + 1e-18) {
                k.bp_head++;
                k.crossed_src_bp = true;
            }
            k.step_count++;
            k.tried_delmin = false;
            if (k.steps_after_bp < kNoRecentBreakpoint) ++k.steps_after_bp;
            if (k.crossed_src_bp && k.step_count > 2) {
                k.steps_after_bp = 0;
                k.order = 1;
                const double gap = (k.bp_head < td.n_bps) ? bp[k.bp_head] - k.time : o.tstop - k.time;
                k.dt = fmin(k.dt, o.restart_scale * fmin(k.saved_delta, gap));
                k.dt = fmax(k.dt, o.dt_min * 2.0);
            }
            if (k.order_cooldown > 0) --k.order_cooldown;
            ctx.order = 2;  // for the promotion test below
        }
        __syncthreads();
        const bool try_promote = (k.order == 1 && k.step_count >= 2 && k.order_cooldown == 0);
        double dt2 = 1e30;
        if (try_promote) dt2 = min_trunc(v, ctx, o, s_red);
        if (threadIdx.x == 0) {
            if (try_promote && dt2 > 1.05 * k.dt) k.order = 2;
            ctx.order = k.order;
        }
        // rotate_state (circuit.cpp:328): state3 <- state2 <- state1, state1 = state0
        __syncthreads();
        {   // every thread rotates its own copy of the pointers
            double* t3 = v.st[3];
            v.st[3] = v.st[2];
            v.st[2] = v.st[1];
            v.st[1] = t3;
        }
        for (int32_t i = threadIdx.x; i < d.n_states; i += blockDim.x) v.st[1][i] = v.st[0][i];
        store_point(v, td, o, probes, times, values, &k, k.time, v.x);
        // history ring: the oldest buffer takes the solution
        for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) sol_prev3[i] = v.x[i];
        __syncthreads();
        if (threadIdx.x == 0) {
            k.points++;
            const int h3 = s_hist[2];
            s_hist[2] = s_hist[1];
            s_hist[1] = s_hist[0];
            s_hist[0] = h3;
            s_ring = 0;
        }
        __syncthreads();
        // Ringing detection (detect_and_handle_ringing, transient.cpp:580-606).
        const bool check = (k.step_count >= 3 && !o.use_gear && k.steps_after_bp >= kRingingMinStepsAfterBp);
        if (check) {
            const double* s = v.x;
            const double* p1 = hist + s_hist[0] * v.n;
            const double* p2 = hist + s_hist[1] * v.n;
            const double* p3 = hist + s_hist[2] * v.n;
            for (int32_t i = threadIdx.x; i < v.num_nodes; i += blockDim.x) {
                const double d2c = s[i] - 2.0 * p1[i] + p2[i];
                const double d2p = p1[i] - 2.0 * p2[i] + p3[i];
                const double tol = o.nopt.reltol * fabs(s[i]) + o.nopt.vntol;
                if (d2c * d2p < 0.0 && fabs(d2c) > tol && fabs(d2p) > tol) {
                    const double d1c = s[i] - p1[i];
                    const double d1p = p1[i] - p2[i];
                    double d1max = fmax(fabs(d1c), fabs(d1p));
                    if (d1max < 1e-30) d1max = 1e-30;
                    if (fmax(fabs(d2c), fabs(d2p)) / d1max > 0.5) s_ring = 1;
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            if (check) {
                k.ringing = (s_ring != 0);
                if (k.ringing) k.ringing_cooldown = 3;
                else if (k.ringing_cooldown > 0) --k.ringing_cooldown;  // tick_cooldown
                ctx.method = (k.ringing || k.ringing_cooldown > 0) ? 1 : 0;
            }
            if (k.step_count >= kLteMinStepCount) {
                double proposed = k.device_dt;
                proposed = fmin(proposed, kMaxDtGrowthFactor * k.dt);
                k.dt = fmax(proposed, o.dt_min);
            }
        }
        __syncthreads();
    }

    __syncthreads();
    if (threadIdx.x == 0) {
        status[d.index] = k.status;
        npoints[d.index] = k.points < o.max_points ? k.points : o.max_points;
        stats[4 * d.index] = k.step_count;
        stats[4 * d.index + 1] = k.rejected;
        stats[4 * d.index + 2] = k.newton_iters;
        stats[4 * d.index + 3] = 0;
    }
}

size_t tran_smem_bytes(int max_col, int max_n) {
    const int colbuf = (max_col + 31) & ~31;
    const size_t a = flow_smem_bytes(colbuf, max_n);
    const size_t b = flow_solve_smem_bytes(max_n);
    return a > b ? a : b;
}

cudaError_t launch_transient(const PlanDesc* plans, const int32_t* lu_pool, const DcDesc* descs,
                             const TranDesc* tdescs, int count, const int32_t* prog,
                             const double* params_dc, const double* params_tran, double* work,
                             const double* bps, const int32_t* probes, double* times,
                             double* values, int32_t* npoints, int32_t* status, int32_t* stats,
                             const TranOptions& o, int max_col, int max_n, cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    const int colbuf = (max_col + 31) & ~31;
    const size_t smem = tran_smem_bytes(max_col, max_n);
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(transient_kernel,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             200 * 1024);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    transient_kernel<<<count, kFlowThreads, smem, stream>>>(
        plans, lu_pool, descs, tdescs, prog, params_dc, params_tran, work, bps, probes, times,
        values, npoints, status, stats, o, colbuf);
    return cudaGetLastError();
}

}  // namespace nsg
