// DC operating point of one instance with the reference's continuation
// aids, as a resumable state machine: the direct Newton attempt, then true
// gmin stepping (device gmin, solve_dc only) and diagonal gmin stepping
// (true_gmin_stepping / gmin_stepping, src/core/convergence.cpp:216-469,
// called from solve_dc, src/core/dc.cpp:53-175, and from the transient's
// compute_dc_operating_point, src/core/transient.cpp:145-205).
//
// The controller lives in global memory (DcCtl) so that an instance whose
// pivots fail re-validation can stop (kStatusReorder), be re-ordered on the
// host, and continue in a later launch exactly where it stopped.
#pragma once
#include "newton_common.cuh"

namespace nsg {

// Save area: x (n), state0..2 (3 n_states).
__device__ inline void dc_op_copy(const Inst& v, int32_t n_states, double* save, int action) {
    if (action == kActNone) return;
    double* sx = save;
    double* ss = save + v.n;
    const int64_t ns3 = 3 * static_cast<int64_t>(n_states);
    if (action == kActZeroSave) {
        for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) v.x[i] = sx[i] = 0.0;
        for (int64_t i = threadIdx.x; i < ns3; i += blockDim.x)
            v.st[i / n_states][i % n_states] = ss[i] = 0.0;
    } else if (action == kActSave) {
        for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) sx[i] = v.x[i];
        for (int64_t i = threadIdx.x; i < ns3; i += blockDim.x) ss[i] = v.st[i / n_states][i % n_states];
    } else {
        for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) v.x[i] = sx[i];
        for (int64_t i = threadIdx.x; i < ns3; i += blockDim.x) v.st[i / n_states][i % n_states] = ss[i];
    }
}

__host__ __device__ inline void dc_op_start(DcCtl* c, int firstmode) {
    c->phase = kOpDirect;
    c->total = 0;
    c->code = kDcNoConvergence;
    c->ctx_mode = firstmode;
    c->active = 0;
    c->action = kActNone;
    c->solves = 0;
    c->method = 0;
}

// Thread 0: start a stepping method from a zero guess and cleared states.
__device__ inline void dc_op_begin_stepping(DcCtl* c, int phase, int firstmode) {
    c->phase = phase;
    c->factor = 10.0;
    c->old = 1e-2;
    c->cur = c->old / c->factor;
    c->total = 0;
    c->ctx_mode = firstmode;
    c->action = kActZeroSave;
}

// Runs the operating point from the controller's current phase.  Returns
// kDcConverged, kDcNoConvergence, kStatusReorder (stopped for the host) or
// kStatusTimeout.  x holds the solution on kDcConverged.  All threads of the
// CTA call it; ctl is read only after barriers and written by thread 0.
__device__ inline int32_t dc_operating_point(const Inst& v, int32_t n_states, const PlanDesc& pd,
                                             const int32_t* lu_pool, IntegCtx* ctx,
                                             SolverState* solver, DcCtl* ctl,
                                             const NewtonOptions& opt, int firstmode,
                                             int contmode, bool true_gmin_first, double* save,
                                             double* smem, int colbuf, int smem_doubles) {
    const double gtarget = opt.gmin;  // max(gmin, gshunt = 0)
    const int itl2 = 50;
    // Bound on Newton solves per operating point: a stepping that creeps by
    // the minimum factor would otherwise run for hours.
    constexpr int kMaxSolves = 20000;
    __shared__ int32_t s_phase, s_active, s_r_iter, s_r_devconv, s_entry_mode, s_action, s_code;
    __shared__ double s_cur;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) {
            s_phase = ctl->phase;
            s_code = ctl->code;
            s_active = ctl->active;
            s_r_iter = ctl->r_iter;
            s_r_devconv = ctl->r_devconv;
            s_entry_mode = ctl->ctx_mode;
            s_cur = ctl->cur;
            ctx->mode = ctl->active ? ctl->r_mode : ctl->ctx_mode;
        }
        __syncthreads();
        const int phase = s_phase;
        if (phase == kOpDone) return s_code;
        NewtonOptions o = opt;
        int max_iter = opt.max_iter;
        if (phase == kOpTrueGmin) {
            o.gmin = s_cur;
            max_iter = itl2 > 100 ? itl2 : 100;
        } else if (phase == kOpDiagGmin) {
            o.diag_gmin = s_cur;
            max_iter = itl2 > 100 ? itl2 : 100;
        } else if (phase == kOpDiagGminFinal) {
            o.diag_gmin = 0.0;
        }
        load_constants(v, o.gmin);  // the dead-node pin follows SimOptions::gmin
        const bool resume = s_active != 0;
        const NewtonOutcome r = newton(v, pd, lu_pool, ctx, o, max_iter, solver, smem, colbuf,
                                       resume ? s_r_iter : -1, s_entry_mode,
                                       resume ? s_r_devconv : 1, false, smem_doubles);
        if (r.code == kStatusReorder) {
            if (threadIdx.x == 0) {
                ctl->active = 1;
                ctl->r_iter = r.fail_iter;
                ctl->r_mode = r.fail_mode;
                ctl->r_devconv = r.fail_dev_conv;
                ctl->numeric_diag_gmin = o.diag_gmin;
            }
            __syncthreads();
            return kStatusReorder;
        }
        if (r.code == kStatusTimeout) return kStatusTimeout;
        const bool conv = (r.code == kDcConverged);
        if (threadIdx.x == 0) {
            DcCtl& c = *ctl;
            c.active = 0;
            c.action = kActNone;
            c.method = (phase == kOpDirect) ? 0 : 1;  // DIRECT / GMIN_STEPPING
            const bool final_ok = conv && (phase == kOpDirect || phase == kOpTrueGminFinal ||
                                           phase == kOpDiagGminFinal);
            if (++c.solves >= kMaxSolves && !final_ok) {
                c.code = kDcNoConvergence;
                c.phase = kOpDone;
            } else if (phase == kOpDirect) {
                if (conv) {
                    c.total = r.iters;
                    c.code = kDcConverged;
                    c.phase = kOpDone;
                } else {
                    dc_op_begin_stepping(&c, true_gmin_first ? kOpTrueGmin : kOpDiagGmin, firstmode);
                }
            } else if (phase == kOpTrueGmin || phase == kOpDiagGmin) {
                c.total += r.iters;
                if (conv) {
                    c.ctx_mode = contmode;
                    if (c.cur <= gtarget) {
                        c.phase = phase + 1;  // the final solve at the target
                    } else {
                        c.action = kActSave;
                        if (r.iters <= itl2 / 4) {
                            c.factor *= sqrt(c.factor);
                            if (c.factor > 10.0) c.factor = 10.0;
                        }
                        if (r.iters > (3 * itl2 / 4)) {
                            const double sq = sqrt(c.factor);
                            c.factor = (sq < 1.00005) ? 1.00005 : sq;
                        }
                        c.old = c.cur;
                        if (c.cur < c.factor * gtarget) {
                            c.factor = c.cur / gtarget;
                            c.cur = gtarget;
                        } else {
                            c.cur /= c.factor;
                        }
                    }
                } else if (c.factor < 1.00005) {
                    if (phase == kOpTrueGmin) {
                        dc_op_begin_stepping(&c, kOpDiagGmin, firstmode);
                    } else {
                        c.code = kDcNoConvergence;
                        c.phase = kOpDone;
                    }
                } else {
                    c.factor = sqrt(sqrt(c.factor));
                    c.cur = c.old / c.factor;
                    c.action = kActRestore;
                }
            } else {  // a final solve at the target gmin
                if (conv) {
                    c.total += r.iters;
                    c.code = kDcConverged;
                    c.phase = kOpDone;
                } else if (phase == kOpTrueGminFinal) {
                    dc_op_begin_stepping(&c, kOpDiagGmin, firstmode);
                } else {
                    c.code = kDcNoConvergence;
                    c.phase = kOpDone;
                }
            }
            s_action = c.action;
        }
        __syncthreads();
        dc_op_copy(v, n_states, save, s_action);
    }
}

}  // namespace nsg
