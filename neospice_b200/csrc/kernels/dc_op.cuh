// DC operating point of one instance with the reference's continuation
// aids, as a resumable state machine: the direct Newton attempt, then true
// gmin stepping (device gmin, solve_dc only) and diagonal gmin stepping
// (true_gmin_stepping / gmin_stepping, src/core/convergence.cpp:216-469),
// source stepping (source_stepping, convergence.cpp:471-581), for solve_dc
// gain stepping (gain_stepping, convergence.cpp:583-703: the same ramp over
// the dependent-source gains, of which this device set has none, so the
// sources stay unscaled), then pseudo-transient continuation
// (pseudo_transient, convergence.cpp:986-1097) — called from solve_dc,
// src/core/dc.cpp:53-242, and from the transient's
// compute_dc_operating_point, src/core/transient.cpp:145-205.
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

// Thread 0: source (gain = 0) or gain (gain = 1) stepping from a zero guess
// and cleared states, starting with the solve at fraction 0.
__host__ __device__ inline void dc_op_begin_source(DcCtl* c, int gain, int firstmode) {
    c->phase = kOpSrcFirst;
    c->gain = gain;
    c->frac = 0.0;
    c->step = 0.001;
    c->next = 0.0;
    c->total = 0;
    c->ctx_mode = firstmode;
    c->action = kActZeroSave;
}

// Thread 0: pseudo-transient continuation from a zero guess and cleared
// states: C = 1e-3, dt = 1e-6, the probe threshold max(1e-6, target * 1e6)
// with the target diag_gmin max(gshunt, 0) = 0.
__host__ __device__ inline void dc_op_begin_ptc(DcCtl* c, int firstmode) {
    c->phase = kOpPtc;
    c->ptc_dt = 1e-6;
    c->ptc_prev = -1.0;
    c->ptc_probe = 1e-6;
    c->ptc_k = 0;
    c->total = 0;
    c->ctx_mode = firstmode;
    c->action = kActZeroSave;
}

// std::min / std::max as the reference evaluates them (the first argument
// wins ties and NaN comparisons).
__host__ __device__ inline double std_min(double a, double b) { return (b < a) ? b : a; }
__host__ __device__ inline double std_max(double a, double b) { return (a < b) ? b : a; }

// first_aid: kAidDirect runs the whole cascade; kAidSource, kAidGain and
// kAidPseudoTransient run source stepping, gain stepping or pseudo-transient
// continuation alone (the instance's x and states are zero then).
__host__ __device__ inline void dc_op_start(DcCtl* c, int firstmode, int first_aid = kAidDirect) {
    c->phase = kOpDirect;
    c->total = 0;
    c->code = kDcNoConvergence;
    c->ctx_mode = firstmode;
    c->active = 0;
    c->action = kActNone;
    c->solves = 0;
    c->method = 0;
    if (first_aid == kAidSource || first_aid == kAidGain) {
        dc_op_begin_source(c, first_aid == kAidGain ? 1 : 0, firstmode);
        c->action = kActNone;
    } else if (first_aid == kAidPseudoTransient) {
        dc_op_begin_ptc(c, firstmode);
        c->action = kActNone;
    }
}

// Thread 0: the next fraction of source stepping (fraction + step, at most 1).
__host__ __device__ inline void dc_op_next_fraction(DcCtl* c) {
    double next = c->frac + c->step;
    if (next > 1.0) next = 1.0;
    c->next = next;
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

// Thread 0, after each Newton solve: the cascade's bookkeeping — the next
// phase, its gmin / fraction / pseudo timestep, the solve count and the
// save / restore action (returned).  Kept out of line: it runs once per
// solve, not per Newton iteration.
static __device__ __noinline__ int32_t dc_op_advance(DcCtl* ctl, int phase, const NewtonOutcome& r,
                                                   bool conv, const NewtonOptions& opt,
                                                   int firstmode, int contmode,
                                                   bool true_gmin_first, double s_ptc_g) {
    const double gtarget = opt.gmin;  // max(gmin, gshunt = 0)
    const int itl2 = 50;
    // Bound on Newton solves per operating point: a stepping that creeps by
    // the minimum factor would otherwise run for hours.
    constexpr int kMaxSolves = 20000;
    DcCtl& c = *ctl;
    c.active = 0;
    c.action = kActNone;
    // DIRECT / GMIN_STEPPING / SOURCE_STEPPING / PSEUDO_TRANSIENT
    // (ConvergenceMethod, src/core/sim_status.hpp:10-17; gain
    // stepping reports SOURCE_STEPPING)
    c.method = (phase == kOpDirect) ? 0
               : (phase >= kOpPtc ? 3 : (phase >= kOpSrcFirst ? 2 : 1));
    const bool final_ok = conv && (phase == kOpDirect || phase == kOpTrueGminFinal ||
                                   phase == kOpDiagGminFinal || phase == kOpPtcProbe ||
                                   phase == kOpPtcFinal ||
                                   (phase == kOpSrcStep && c.next >= 1.0));
    auto fail_all = [&]() {
        c.code = kDcNoConvergence;
        c.phase = kOpDone;
    };
    // After source stepping fails: gain stepping in solve_dc, then
    // pseudo-transient continuation (directly after source stepping
    // in the transient's operating point); the aids after it are not
    // built.  A run started at an aid ends with it.
    auto source_failed = [&]() {
        if (opt.first_aid != kAidDirect) {
            fail_all();
        } else if (true_gmin_first && !c.gain) {
            dc_op_begin_source(&c, 1, firstmode);
        } else {
            dc_op_begin_ptc(&c, firstmode);
        }
    };
    // The pseudo-transient step loop: the next step, or the final
    // attempt after 200 steps.
    auto ptc_next_step = [&]() {
        if (++c.ptc_k >= 200) c.phase = kOpPtcFinal;
        else c.phase = kOpPtc;
    };
    if (++c.solves >= kMaxSolves && !final_ok) {
        fail_all();
    } else if (phase == kOpPtc) {
        if (conv) {
            c.total += r.iters;
            c.action = kActSave;
            c.ctx_mode = contmode;
            const double curr = r.residual;
            if (c.ptc_prev > 0.0 && curr > 0.0) {
                double ratio = c.ptc_prev / curr;
                ratio = std_min(ratio, 4.0);
                ratio = std_max(ratio, 0.25);
                c.ptc_dt *= ratio;
            } else {
                c.ptc_dt *= 2.0;
            }
            c.ptc_dt = std_max(c.ptc_dt, 1e-15);
            c.ptc_dt = std_min(c.ptc_dt, 1e6);
            c.ptc_prev = curr;
            if (s_ptc_g <= c.ptc_probe) {
                c.phase = kOpPtcProbe;  // from the accepted state just saved
            } else {
                ptc_next_step();
            }
        } else {
            c.action = kActRestore;
            c.ptc_dt /= 4.0;
            c.ptc_prev = -1.0;
            if (c.ptc_dt < 1e-15) c.phase = kOpPtcFinal;
            else ptc_next_step();
        }
    } else if (phase == kOpPtcProbe) {
        if (conv) {
            c.total += r.iters;
            c.code = kDcConverged;
            c.phase = kOpDone;
        } else {
            c.action = kActRestore;  // the probe's start = the accepted state
            c.ptc_probe *= 1e-3;
            ptc_next_step();
        }
    } else if (phase == kOpPtcFinal) {
        if (conv) {
            c.total += r.iters;
            c.code = kDcConverged;
        } else {
            c.code = kDcNoConvergence;
        }
        c.phase = kOpDone;
    } else if (phase == kOpSrcFirst) {
        c.r0_iters = r.iters;
        if (conv) {
            c.total += r.iters;
            c.action = kActSave;
            c.ctx_mode = contmode;
            c.phase = kOpSrcStep;
            dc_op_next_fraction(&c);
        } else {
            // gmin ramp at zero sources: diag_gmin from gmin * 10^10
            double diag = opt.gmin;
            for (int i = 0; i < 10; ++i) diag *= 10.0;
            c.zdiag = diag;
            c.zi = 0;
            c.action = kActZeroSave;
            c.ctx_mode = firstmode;
            c.phase = kOpSrcZeroGmin;
        }
    } else if (phase == kOpSrcZeroGmin) {
        if (!conv) {
            source_failed();
        } else {
            c.total += r.iters;
            c.zdiag /= 10.0;
            c.ctx_mode = contmode;
            if (c.zi == 10) {
                c.total += c.r0_iters;  // the failed solve at zero sources
                c.action = kActSave;
                c.phase = kOpSrcStep;
                dc_op_next_fraction(&c);
            } else {
                ++c.zi;
            }
        }
    } else if (phase == kOpSrcStep) {
        const int quarter = opt.max_iter / 4, half = opt.max_iter / 2;
        if (conv) {
            c.total += r.iters;
            c.frac = c.next;
            c.action = kActSave;
            if (r.iters < quarter) {
                const double s = c.step * 1.5;
                c.step = (s < 0.1) ? s : 0.1;
            } else if (r.iters > half) {
                const double s = c.step * 0.5;
                c.step = (1e-7 < s) ? s : 1e-7;
            }
            if (c.frac < 1.0) {
                dc_op_next_fraction(&c);
            } else {
                c.code = kDcConverged;
                c.phase = kOpDone;
            }
        } else if (c.step * (1.0 - c.frac) < 1e-8) {
            source_failed();
        } else {
            c.action = kActRestore;
            c.step *= 0.1;
            if (c.step > 0.01) c.step = 0.01;
            if (c.step < 1e-7) {
                source_failed();
            } else {
                dc_op_next_fraction(&c);
            }
        }
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
                dc_op_begin_source(&c, 0, firstmode);
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
            dc_op_begin_source(&c, 0, firstmode);
        }
    }
    return c.action;
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
    const int itl2 = 50;
    __shared__ int32_t s_phase, s_active, s_r_iter, s_r_devconv, s_entry_mode, s_action, s_code;
    __shared__ int32_t s_gain;
    __shared__ double s_cur, s_next, s_zdiag, s_ptc_g;
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
            s_gain = ctl->gain;
            s_next = ctl->next;
            s_zdiag = ctl->zdiag;
            s_ptc_g = 1e-3 / ctl->ptc_dt;  // C_pseudo / dt_pseudo
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
        } else if (phase >= kOpSrcFirst) {
            // SimOptions::src_fact at 0, then the fraction under solve; the
            // zero-source ramp adds its diag_gmin.  Gain stepping leaves the
            // sources at full value.
            if (phase >= kOpPtc) {
                // diag_gmin = target + C/dt on a step, the target (0) on the
                // probe and the final attempt; at most 100 iterations
                o.diag_gmin = (phase == kOpPtc) ? 0.0 + s_ptc_g : 0.0;
                o.want_residual = 1;
                max_iter = opt.max_iter < 100 ? opt.max_iter : 100;
            } else {
                if (!s_gain) o.src_fact = (phase == kOpSrcStep) ? s_next : 0.0;
                if (phase == kOpSrcZeroGmin) o.diag_gmin = s_zdiag;
            }
        }
        load_constants(v, o.gmin, o.src_fact);  // the dead-node pin follows SimOptions::gmin
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
        if (threadIdx.x == 0)
            s_action = dc_op_advance(ctl, phase, r, conv, opt, firstmode, contmode,
                                     true_gmin_first, s_ptc_g);
        __syncthreads();
        dc_op_copy(v, n_states, save, s_action);
    }
}

}  // namespace nsg
