// Per-instance Newton machinery shared by the DC and transient kernels: one
// CTA (kFlowThreads threads) owns one circuit instance.
#pragma once
#include "dc_device.cuh"
#include "diode_model.cuh"
#include "lu_cta.cuh"
#include "bsim4_model.cuh"
#include "mos1_model.cuh"
#include "source_wave.cuh"

namespace nsg {

// CKTmode bits (ngspice cktdefs.h, as used in src/core/newton.cpp:109-115,
// src/devices/capacitor.cpp:37-44).
constexpr int kModeTran = 0x1;
constexpr int kModeAc = 0x2;
constexpr int kModeDcOp = 0x10;
constexpr int kModeTranOp = 0x20;
constexpr int kModeDcMask = 0x70;
constexpr int kModeInitFloat = 0x100;
constexpr int kModeInitJct = 0x200;
constexpr int kModeInitFix = 0x400;
constexpr int kModeInitTran = 0x1000;
constexpr int kModeInitPred = 0x2000;
constexpr int kModeUic = 0x10000;
constexpr int kModeInitMask = 0x3F00;

// Views of one instance's program and workspace.
struct Inst {
    const int32_t* slot_ptr;
    const int32_t* slot_terms;
    const int32_t* rhs_ptr;
    const int32_t* rhs_terms;
    const int32_t* ucb_ptr;
    const int32_t* ucb_terms;
    const int32_t* term_op;
    const int32_t* term_param;
    const int32_t* diodes;  // (pos, neg, param, state)
    const int32_t* caps;    // (pos, neg, param, has_ic, state)
    const int32_t* srcs;    // (is_voltage, wave, param, nparam)
    const int32_t* mos;     // (d, g, s, b, param, state, family): level 1 or BSIM4v7
    const double* par;
    double* x;
    double* xold;
    double* a;
    double* lu;
    double* lrows;
    double* urows;
    double* tv;
    double* dconst;
    double* st[4];          // device state ring state0..state3
    double* mrec;           // per-MOSFET load values (kMosRecCount each)
    int32_t n, num_nodes, nnz, n_const, n_diodes, n_caps, n_srcs, n_mos;
    int32_t* rmaps = nullptr;  // optional row -> position maps of the CTA's warps
    int64_t rmap_stride = 0;   // words per warp
};

// Address of workspace offset `off`: in the shared-memory stage when the
// instance is staged and the offset lies in its staged span, else global.
__device__ __forceinline__ double* ws_at(const DcDesc& d, double* work, double* stage,
                                         int64_t off) {
    return (stage && off >= d.x_off && off < d.x_off + d.stage_len) ? stage + (off - d.x_off)
                                                                     : work + off;
}

// Copy the staged span between global memory and the stage (whole CTA).
__device__ inline void stage_copy(const DcDesc& d, double* work, double* stage, bool in) {
    if (!stage) return;
    __syncthreads();
    double* g = work + d.x_off;
    for (int64_t i = threadIdx.x; i < d.stage_len; i += blockDim.x) {
        if (in) stage[i] = g[i];
        else g[i] = stage[i];
    }
    __syncthreads();
}

__device__ inline Inst make_inst(const DcDesc& d, const int32_t* prog, const double* params,
                                 double* work, double* stage = nullptr) {
    Inst v;
    v.slot_ptr = prog + d.prog_off[DP_slot_ptr];
    v.slot_terms = prog + d.prog_off[DP_slot_terms];
    v.rhs_ptr = prog + d.prog_off[DP_rhs_ptr];
    v.rhs_terms = prog + d.prog_off[DP_rhs_terms];
    v.ucb_ptr = prog + d.prog_off[DP_ucb_ptr];
    v.ucb_terms = prog + d.prog_off[DP_ucb_terms];
    v.term_op = prog + d.prog_off[DP_term_op];
    v.term_param = prog + d.prog_off[DP_term_param];
    v.diodes = prog + d.prog_off[DP_diodes];
    v.caps = prog + d.prog_off[DP_caps];
    v.srcs = prog + d.prog_off[DP_srcs];
    v.mos = prog + d.prog_off[DP_mos];
    v.par = params + d.param_off;
    v.x = ws_at(d, work, stage, d.x_off);
    v.xold = ws_at(d, work, stage, d.xold_off);
    v.a = ws_at(d, work, stage, d.a_off);
    v.lu = ws_at(d, work, stage, d.lu_off);
    v.lrows = ws_at(d, work, stage, d.lrows_off);
    v.urows = ws_at(d, work, stage, d.urows_off);
    v.tv = ws_at(d, work, stage, d.tv_off);
    v.dconst = ws_at(d, work, stage, d.dconst_off);
    for (int k = 0; k < 4; ++k)
        v.st[k] = ws_at(d, work, stage, d.state_off) + k * static_cast<int64_t>(d.n_states);
    v.n = d.n;
    v.num_nodes = d.num_nodes;
    v.nnz = d.nnz;
    v.n_const = d.n_const;
    v.n_diodes = d.n_diodes;
    v.n_caps = d.n_caps;
    v.n_srcs = d.n_srcs;
    v.n_mos = d.n_mos;
    v.mrec = ws_at(d, work, stage, d.mrec_off);
    return v;
}

__device__ __forceinline__ double term_value(int32_t op, double p, double gmin) {
    switch (op) {
        case 0: return 1.0 / p;
        case 1: return -(1.0 / p);
        case 2: return p;
        case 3: return -p;
        case 4: return 1.0;
        case 5: return -1.0;
        case 6: return 0.0;
        case 7: return -0.0;
        default: return gmin;
    }
}

// Constant term values, diode constants (csat, vte, Vcrit at the diode's
// temperature).
// DC source values are scaled by src_fact as VSource / ISource::evaluate do
// (vsource.cpp:208-209, isource.cpp:173-176): the value times the factor,
// then its negation where the stamp subtracts it.
__device__ inline void load_constants(const Inst& v, double gmin, double src_fact = 1.0) {
    for (int32_t k = threadIdx.x; k < v.n_const; k += blockDim.x) {
        const int32_t pi = v.term_param[k];
        const int32_t op = v.term_op[k];
        const double p = pi >= 0 ? v.par[pi] : 0.0;
        v.tv[k] = (op == 2) ? p * src_fact : (op == 3) ? -(p * src_fact) : term_value(op, p, gmin);
    }
    for (int32_t k = threadIdx.x; k < v.n_diodes; k += blockDim.x) {
        const int32_t pi = v.diodes[4 * k + 2];
        const double csat = v.par[pi];
        const double vte = v.par[pi + 1] * v.par[pi + kDpVt];
        v.dconst[3 * k] = csat;
        v.dconst[3 * k + 1] = vte;
        v.dconst[3 * k + 2] = diode_vcrit(vte, csat);
    }
}

// NIintegrate of the charge in state slot q (its current in q + 1):
// backward Euler at order 1, else trapezoidal (xmu_ratio) or Gear-2
// (src/devices/dio/dio_shim.cpp:44-73).  Returns the current.
__device__ inline double ni_integrate(const Inst& v, const IntegCtx& c, int32_t q) {
    const int order = c.order < 1 ? 1 : (c.order > 2 ? 2 : c.order);
    const double* s0 = v.st[0];
    const double* s1 = v.st[1];
    double deriv;
    if (order == 1) deriv = c.ag[0] * s0[q] + c.ag[1] * s1[q];
    else if (c.method == 0) deriv = -s1[q + 1] * c.xmu_ratio + c.ag[0] * s0[q] + c.ag[1] * s1[q];
    else deriv = c.ag[0] * s0[q] + c.ag[1] * s1[q] + c.ag[2] * v.st[2][q];
    v.st[0][q + 1] = deriv;
    return deriv;
}

// Device loads of one Newton iteration at the guess xold: diodes (DIOload
// with its charge storage), capacitors (Capacitor::evaluate, state-vector
// path), MOSFETs, waveform sources (value_at).  Writes the dynamic terms; returns through s_dev_conv
// whether every device reports convergence (diodes' CKTnoncon and conv_test).
// BSIM4v7 load out of line: its few hundred live values get their own
// register allocation instead of spilling eval_devices' loop state.
static __device__ __noinline__ void bsim4_load_call(const double* P, double* rec, double* s0,
                                                    double* s1, const double* s2, int mode,
                                                    const Mos1Integ& ic, const NewtonOptions& opt,
                                                    const double* vn, double* t) {
    bsim4_load(P, rec, s0, s1, s2, mode, ic, opt.gmin, opt.reltol, opt.abstol, vn, t);
}

static __device__ __noinline__ void eval_devices(const Inst& v, const IntegCtx& c, const NewtonOptions& opt,
                                    int32_t* s_dev_conv) {
    const int mode = c.mode;
    double* tv_d = v.tv + v.n_const;
    double* tv_c = tv_d + kDiodeTermCount * v.n_diodes;
    double* tv_s = tv_c + kCapTermCount * v.n_caps;
    const bool uic_op = (mode & kModeTranOp) && (mode & kModeUic);
    const bool charges = (mode & (kModeTran | kModeAc)) || uic_op;
    for (int32_t k = threadIdx.x; k < v.n_diodes; k += blockDim.x) {
        const int32_t* dr = v.diodes + 4 * k;
        const int32_t pos = dr[0], neg = dr[1], s = dr[3];
        const double vp = pos >= 0 ? v.xold[pos] : 0.0;
        const double vn = neg >= 0 ? v.xold[neg] : 0.0;
        double* s0 = v.st[0] + s;
        double* s1 = v.st[1] + s;
        // The junction voltage of this load (dio_load.cpp:100-166; no OFF,
        // IC = 0).
        double vd = vp - vn;
        bool limit = false;
        if (mode & kModeInitTran) {
            vd = s1[kDsV];
        } else if ((mode & kModeInitJct) && uic_op) {
            vd = 0.0;
        } else if (mode & kModeInitJct) {
            vd = v.dconst[3 * k + 2];
        } else {
            if (mode & kModeInitPred) {  // DEVpred
                s0[kDsV] = s1[kDsV];
                const double xfact = c.delta / c.delta_old[1];
                vd = ((1.0 + xfact) * s1[kDsV]) - (xfact * v.st[2][s + kDsV]);
                s0[kDsI] = s1[kDsI];
                s0[kDsG] = s1[kDsG];
            }
            limit = true;
        }
        const DiodeDC r = diode_eval(vd, limit, s0[kDsV], v.dconst[3 * k], v.dconst[3 * k + 1],
                                     v.dconst[3 * k + 2], opt.gmin,
                                     diode_brk(v.par + dr[2], v.par[dr[2] + kDpVt]));
        double cd = r.cd, gd = r.gd;
        if (charges) {  // charge storage (dio_load.cpp:309-373)
            double charge, capd;
            diode_charge(v.par + dr[2], r.vd, r.cdb, r.gdb, &charge, &capd);
            s0[kDsQ] = charge;
            if (!uic_op) {
                if (mode & kModeInitTran) s1[kDsQ] = s0[kDsQ];
                const double ccap = ni_integrate(v, c, s + kDsQ);
                gd = gd + c.ag[0] * capd;
                cd = cd + ccap;
                if (mode & kModeInitTran) s1[kDsCq] = s0[kDsCq];
            }
        }
        s0[kDsV] = r.vd;
        s0[kDsI] = cd;
        s0[kDsG] = gd;
        const double cdeq = cd - gd * r.vd;
        double* t = tv_d + kDiodeTermCount * k;
        t[0] = gd;
        t[1] = gd + diode_gspr(v.par + dr[2]);
        t[2] = -gd;
        t[3] = cdeq;
        t[4] = -cdeq;
        // DIODevice::conv_test (dio_device.cpp:296-307) on the stored state
        const double delvd = (vp - vn) - r.vd;
        const double cdhat = cd + gd * delvd;
        const double tol = opt.reltol * fmax(fabs(cdhat), fabs(cd)) + opt.abstol;
        if (!((r.check == 0) && (fabs(cdhat - cd) <= tol))) *s_dev_conv = 0;
    }
    for (int32_t k = threadIdx.x; k < v.n_caps; k += blockDim.x) {
        const int32_t* cr = v.caps + 5 * k;
        const double cap = v.par[cr[2]];
        double* t = tv_c + kCapTermCount * k;
        const int32_t s = cr[4];  // {q, i} at s, s+1
        if (!(mode & (kModeTran | kModeAc | kModeTranOp))) {
            t[0] = t[1] = t[2] = t[3] = 0.0;
            continue;
        }
        const bool cond1 = ((mode & kModeDcMask) && (mode & kModeInitJct)) ||
                           ((mode & kModeUic) && (mode & kModeInitTran));
        double vcap;
        if (cond1) {
            vcap = cr[3] ? v.par[cr[2] + 1] : 0.0;
        } else {
            const double vp = cr[0] >= 0 ? v.xold[cr[0]] : 0.0;
            const double vn = cr[1] >= 0 ? v.xold[cr[1]] : 0.0;
            vcap = vp - vn;
        }
        if (mode & (kModeTran | kModeAc)) {
            double* s0 = v.st[0];
            double* s1 = v.st[1];
            if (mode & kModeInitPred) {
                s0[s] = s1[s];
            } else {
                s0[s] = cap * vcap;
                if (mode & kModeInitTran) s1[s] = s0[s];
            }
            int order = c.order < 1 ? 1 : (c.order > 2 ? 2 : c.order);
            double deriv;
            if (order == 1) {
                deriv = c.ag[0] * s0[s] + c.ag[1] * s1[s];
            } else if (c.method == 0) {
                deriv = -s1[s + 1] * c.xmu_ratio + c.ag[0] * s0[s] + c.ag[1] * s1[s];
            } else {
                deriv = c.ag[0] * s0[s] + c.ag[1] * s1[s] + c.ag[2] * v.st[2][s];
            }
            s0[s + 1] = deriv;
            const double geq = c.ag[0] * cap;
            const double ceq = s0[s + 1] - c.ag[0] * s0[s];
            if (mode & kModeInitTran) s1[s + 1] = s0[s + 1];
            t[0] = 1.0 * geq;
            t[1] = -1.0 * geq;
            t[2] = -1.0 * ceq;
            t[3] = 1.0 * ceq;
        } else {
            v.st[0][s] = cap * vcap;
            t[0] = t[1] = t[2] = t[3] = 0.0;
        }
    }
    double* tv_m = tv_s + kSrcTermCount * v.n_srcs;
    if (v.n_mos > 0) {
        const Mos1Integ ic{c.ag[0], c.ag[1], c.ag[2], c.xmu_ratio, c.delta, c.delta_old[1],
                           c.order, c.method};
        for (int32_t k = threadIdx.x; k < v.n_mos; k += blockDim.x) {
            const int32_t* mr = v.mos + kMosTabStride * k;
            double vn[4];
            for (int q = 0; q < 4; ++q) vn[q] = mr[q] >= 0 ? v.xold[mr[q]] : 0.0;
            const int32_t s = mr[5];
            if (mr[6] == kMosFamilyBsim4)
                bsim4_load_call(v.par + mr[4], v.mrec + kMosRecCount * k, v.st[0] + s,
                                v.st[1] + s, v.st[2] + s, mode, ic, opt, vn,
                                tv_m + kMosTermCount * k);
            else
                mos1_load(v.par + mr[4], v.mrec + kMosRecCount * k, v.st[0] + s, v.st[1] + s,
                          v.st[2] + s, mode, ic, opt.gmin, vn, tv_m + kMosTermCount * k);
        }
    }
    for (int32_t k = threadIdx.x; k < v.n_srcs; k += blockDim.x) {
        const int32_t* sr = v.srcs + 4 * k;
        const double val = wave_value(sr[1], v.par + sr[2], sr[3], c.time) * opt.src_fact;
        tv_s[kSrcTermCount * k] = val;
        tv_s[kSrcTermCount * k + 1] = -val;
    }
}

// Matrix values and rhs (into x) from the stamp program, in load order.
__device__ inline void assemble(const Inst& v) {
    for (int32_t s = threadIdx.x; s < v.nnz; s += blockDim.x) {
        double acc = 0.0;
        for (int32_t k = v.slot_ptr[s]; k < v.slot_ptr[s + 1]; ++k)
            acc = __dadd_rn(acc, v.tv[v.slot_terms[k]]);
        v.a[s] = acc;
    }
    for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) {
        double nat = 0.0, ucb = 0.0;
        for (int32_t k = v.rhs_ptr[i]; k < v.rhs_ptr[i + 1]; ++k) nat = __dadd_rn(nat, v.tv[v.rhs_terms[k]]);
        for (int32_t k = v.ucb_ptr[i]; k < v.ucb_ptr[i + 1]; ++k) ucb = __dadd_rn(ucb, v.tv[v.ucb_terms[k]]);
        v.x[i] = __dadd_rn(nat, ucb);
    }
}

// Shared memory reserved for a staged plan (stage_plan) by the kernels that
// run many Newton iterations per launch on small instances.
constexpr size_t kPlanStageBytes = 16 * 1024;

// Copy a plan's index arrays into shared memory (whole CTA) when the
// instance takes the shared-memory LU path (n <= 128) and the arrays fit
// cap_words: the refactor and the sweeps read them every Newton iteration,
// thousands of times per launch in a transient.  Returns the pool to read
// the plan from; *out (shared) receives the plan descriptor rebased on it.
// Begins and ends with __syncthreads().
__device__ inline const int32_t* stage_plan(const PlanDesc& pd, const int32_t* pool, int32_t* sm,
                                            int64_t cap_words, PlanDesc* out) {
    const bool fit = sm && pd.n <= 128 && pd.words > 0 && pd.words <= cap_words;
    __syncthreads();
    if (threadIdx.x == 0) {
        *out = pd;
        if (fit)
            for (int k = 0; k < PA_COUNT; ++k) out->off[k] -= pd.off[0];
    }
    if (fit)
        for (int64_t i = threadIdx.x; i < pd.words; i += blockDim.x) sm[i] = pool[pd.off[0] + i];
    __syncthreads();
    return fit ? sm : pool;
}

struct NewtonOutcome {
    int32_t code;       // kDcConverged, kDcNoConvergence, kStatus*
    int32_t iters;
    int32_t fail_iter;  // kStatusReorder / kStatusNeedOrder: the 0-based iteration that stopped,
    int32_t fail_mode;  // the mode it ran in
    int32_t fail_dev_conv;  // and its device-load convergence verdict
    double residual;        // opt.want_residual: max |rhs| over the node rows of the last load
};

// newton.cpp:199-208: the largest |rhs[i]| over the node rows of the
// assembled right-hand side (in x, before the solve overwrites it); a NaN
// row never wins.  Whole CTA; every thread gets the value.
static __device__ __noinline__ double rhs_residual(const Inst& v) {
    __shared__ double s_resid[32];
    double m = 0.0;
    for (int32_t i = threadIdx.x; i < v.num_nodes; i += blockDim.x) {
        const double r = fabs(v.x[i]);
        if (r > m) m = r;
    }
    for (int off = 16; off > 0; off >>= 1) {
        const double o = __shfl_xor_sync(0xffffffffu, m, off);
        if (o > m) m = o;
    }
    if ((threadIdx.x & 31) == 0) s_resid[threadIdx.x >> 5] = m;
    __syncthreads();
    m = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w)
        if (s_resid[w] > m) m = s_resid[w];
    __syncthreads();
    return m;
}

// newton_solve (src/core/newton.cpp:51-419) for the whole CTA: x holds the
// initial guess and receives the solution (the previous iterate on
// convergence).  *ctx is the instance's integrator context (mode updated in
// place, restored to saved_mode on exit).
//
// A numeric() whose pivot re-validation fails (NeoSolver would re-order on
// the host) ends the call with kStatusReorder, fail_iter, fail_mode and
// fail_dev_conv, the term values of that iteration left in v.tv.  After the
// host has re-ordered on that matrix, calling again with resume_iter =
// fail_iter, resume_dev_conv = fail_dev_conv, ctx->mode = fail_mode and
// saved_mode = the original call's mode continues the same Newton solve: the
// matrix is re-assembled from v.tv (no device re-evaluation) and refactored
// with the new pivots.  With host_orders_first the solver's first numeric()
// stops the same way with kStatusNeedOrder, for the host to order a fresh
// topology on that matrix.  With fixed_pivots every factorization replays the
// plan's pivots unchecked (only a zero pivot fails): for callers that need a
// solution of the equations, not the reference's pivoting (the adjoint's
// re-solves).
__device__ inline NewtonOutcome newton(const Inst& v, const PlanDesc& pd, const int32_t* lu_pool,
                                       IntegCtx* ctx, const NewtonOptions& opt, int max_iter,
                                       SolverState* solver, double* smem, int colbuf,
                                       int resume_iter = -1, int saved_mode = -1,
                                       int resume_dev_conv = 1, bool host_orders_first = false,
                                       int smem_doubles = 0, bool fixed_pivots = false) {
    __shared__ int32_t s_conv, s_dev_conv;
    if (saved_mode < 0) saved_mode = ctx->mode;
    bool force_numeric = false;
    NewtonOutcome out{kDcNoConvergence, max_iter, -1, 0, 1, 0.0};
    double residual = 0.0;
    // Small instances keep the LU in shared memory (warp-level refactor and
    // sweeps); larger ones use the dataflow schedule over global memory.
    const bool small = small_fits(pd.n, pd.nnz_lu, smem_doubles);
    double* lu_s = smem;
    double* w_s = smem + pd.nnz_lu;
    __syncthreads();
    for (int iter = resume_iter < 0 ? 0 : resume_iter; iter < max_iter; ++iter) {
        const bool resumed = (iter == resume_iter);
        if (!resumed) {
            for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) v.xold[i] = v.x[i];
            if (threadIdx.x == 0) s_dev_conv = 1;
            __syncthreads();
            eval_devices(v, *ctx, opt, &s_dev_conv);
        } else if (threadIdx.x == 0) {
            s_dev_conv = resume_dev_conv;  // this iteration's loads ran before the host round trip
        }
        __syncthreads();
        assemble(v);
        __syncthreads();
        if (opt.want_residual) residual = rhs_residual(v);

        const int mode = ctx->mode;
        const bool numeric = resumed || force_numeric || (mode & kModeInitJct) || !solver->factored;
        if (host_orders_first && numeric && !solver->factored && !resumed) {
            out = {kStatusNeedOrder, iter + 1, iter, mode, s_dev_conv};
            break;
        }
        // numeric() on a factored solver re-validates (Markowitz) or
        // re-chooses (AMD-LU) the pivots; refactorize() replays them (AMD-LU
        // with the growth test).  A resumed iteration replays the pivots the
        // host just chose.
        const int check = fixed_pivots ? kCheckNone
                          : numeric ? ((solver->factored && !resumed) ? kCheckNumeric : kCheckNone)
                                    : kCheckRefactor;
        const RefactorResult fr =
            small ? cta_refactor_small(pd, lu_pool, v.a, v.lu, opt.diag_gmin, check, 1e-3, lu_s)
                  : cta_refactor_flow(pd, lu_pool, v.a, v.lu, opt.diag_gmin, check, 1e-3, smem,
                                      colbuf, v.lrows, v.urows, v.rmaps, v.rmap_stride);
        if (fr.code == kStatusTimeout) {
            out = {kStatusTimeout, iter + 1, -1, 0, 1};
            break;
        }
        if (numeric) {
            if (fr.code != kStatusOk) {
                // NeoSolver::numeric would re-order (103) or report singular.
                out = {fr.code, iter + 1, iter, mode, s_dev_conv};
                break;
            }
            if (threadIdx.x == 0) solver->factored = 1;
            force_numeric = false;
        } else if (fr.code == kStatusReorder) {
            // AMD-LU replay failed its growth test: the reference's
            // refactorize() falls back to a full factor_ on this matrix,
            // which the host performs before this iteration resumes.
            out = {fr.code, iter + 1, iter, mode, s_dev_conv};
            break;
        } else if (fr.code != kStatusOk) {
            force_numeric = true;  // newton.cpp:229-234: retry with numeric
            for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) v.x[i] = v.xold[i];
            __syncthreads();
            continue;
        }
        if (small) {
            cta_solve_small(pd, lu_pool, lu_s, v.x, w_s);
        } else if (!cta_solve_flow(pd, lu_pool, v.lu, v.lrows, v.urows, v.x, smem)) {
            out = {kStatusTimeout, iter + 1, -1, 0, 1};
            break;
        }

        // Convergence test (newton.cpp:267-292).
        if (threadIdx.x == 0) s_conv = 1;
        __syncthreads();
        for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) {
            const double vn = v.x[i], vo = v.xold[i];
            bool ok = !(isnan(vn) || isinf(vn));
            if (ok) {
                const double tol = opt.reltol * fmax(fabs(vn), fabs(vo)) +
                                   (i < v.num_nodes ? opt.vntol : opt.abstol);
                ok = fabs(vn - vo) <= tol;
            }
            if (!ok) s_conv = 0;
        }
        __syncthreads();
        if (v.n_mos > 0 && s_conv != 0 && iter > 0) {
            // MOS1Device::device_converged(solution) on the new solution;
            // BSIM4v7Device::device_converged() is the last load's verdict.
            for (int32_t k = threadIdx.x; k < v.n_mos; k += blockDim.x) {
                const int32_t* mr = v.mos + kMosTabStride * k;
                if (mr[6] == kMosFamilyBsim4) {
                    if (v.mrec[kMosRecCount * k + kB4RNoncon] != 0.0) s_dev_conv = 0;
                    continue;
                }
                double vn[4];
                for (int q = 0; q < 4; ++q) vn[q] = mr[q] >= 0 ? v.x[mr[q]] : 0.0;
                if (!mos1_converged(v.par + mr[4], v.mrec + kMosRecCount * k, v.st[0] + mr[5], vn,
                                    opt.reltol, opt.abstol))
                    s_dev_conv = 0;
            }
            __syncthreads();
        }
        const bool conv = (s_conv != 0) && iter > 0 && (s_dev_conv != 0);

        bool done = false;
        if (mode & kModeInitFloat) {
            if (conv) {
                for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) v.x[i] = v.xold[i];
                out = {kDcConverged, iter + 1, -1, 0, 1};
                done = true;
            }
        } else if (mode & kModeInitJct) {
            if (threadIdx.x == 0) ctx->mode = (mode & ~kModeInitMask) | kModeInitFix;
            force_numeric = true;
        } else if (mode & kModeInitFix) {
            if (conv && threadIdx.x == 0) ctx->mode = (mode & ~kModeInitMask) | kModeInitFloat;
        } else if (mode & kModeInitTran) {
            if (threadIdx.x == 0) ctx->mode = (mode & ~kModeInitMask) | kModeInitFloat;
            force_numeric = true;  // NISHOULDREORDER after MODEINITTRAN (newton.cpp:396-399)
        } else if (mode & kModeInitPred) {
            if (threadIdx.x == 0) ctx->mode = (mode & ~kModeInitMask) | kModeInitFloat;
        } else if (conv) {
            for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) v.x[i] = v.xold[i];
            out = {kDcConverged, iter + 1, -1, 0, 1};
            done = true;
        }
        __syncthreads();
        if (done) break;
    }
    __syncthreads();
    if (out.code != kDcConverged && out.code != kDcNoConvergence) {
        // stopped inside the loop: the caller's guess is the last iterate
        for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) v.x[i] = v.xold[i];
    }
    if (threadIdx.x == 0) ctx->mode = saved_mode;
    __syncthreads();
    out.residual = residual;
    return out;
}

}  // namespace nsg
