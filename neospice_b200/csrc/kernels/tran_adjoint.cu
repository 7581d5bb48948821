// Batched transient adjoint: gradients of
//   L = w * sum_n (x_n[probe] - target_n)^2      (n = 0: the operating point)
// through the discrete transient of one instance per CTA, with respect to
// resistances, capacitances and the W, L and VTO of level-1 MOSFETs.
//
// The forward run (transient_kernel with recording on) fixes the timepoints
// and, per accepted step, the integration formula (NIintegrate coefficients,
// order, method).  This kernel replays that schedule -- Newton on each step
// with the plan's pivots -- keeping a checkpoint every K steps, then walks the
// steps backwards, re-solving each K-step segment from its checkpoint.  With
// the capacitor currents i_n = ag0 q_n + ag1 q_{n-1} + ag2 q_{n-2}
// - r i_{n-1} (q = C v; r = xmu/(1-xmu) for the trapezoidal rule, else 0)
// and the step residual R_n = f(x_n) + B i_n - s(t_n), the discrete adjoint
// is, per step from last to first (eta, mu per capacitor):
//   mu_n    = -r_{n+1} eta_{n+1}
//   J_n^T lambda_n = dl_n/dx_n + B (ag0_n C mu_n + ag1_{n+1} C eta_{n+1}
//                                   + ag2_{n+2} C eta_{n+2})
//   eta_n   = mu_n - B^T lambda_n
//   dL/dC  += eta_n (ag0_n v_n + ag1_n v_{n-1} + ag2_n v_{n-2})
//   dL/dp  -= lambda_n^T dR_n/dp      (R, MOSFET W / L / VTO)
// with J_n the Newton matrix at x_n (the forward's own assembly and
// fixed-pivot refactor) and lambda from the transposed solve; the operating
// point closes the recursion with the DC Jacobian.  A diode's charge
// q(v) (depletion plus transit-time charge, a function of its junction
// voltage) enters the same recursion as a capacitor with C replaced by
// dq/dv at the step whose charge it is (q_s appears in i_s, i_{s+1} and
// i_{s+2}); diode parameters are not differentiated.
//
// Level-1 MOSFET charges (mos1_model.cuh) enter as five more units per
// instance.  The bulk junctions are charges q(v) like the diode's.  The
// Meyer gate charges are accumulated, q_n = G_n = q_{n-1} + (v_n - v_{n-1})
// c_n with c_n = h(x_n) + h(x_{n-1}) + overlap, and the current a Meyer
// unit puts into the step residual is I_n = i_n + ag0 q_n (1 - c_n) (the
// charge integration MOS1load calls returns ceq = i - geq q, and the load
// adds ag0 q back), so each unit carries a charge adjoint kappa besides
// eta (beta_n = B^T lambda_n):
//   kappa_n = ag0_n eta_n + ag1_{n+1} eta_{n+1} + ag2_{n+2} eta_{n+2}
//             + kappa_{n+1} - ag0_n (1 - c_n) beta_n
// (dG_n/dx_n)^T kappa_n, (dG_{n+1}/dx_n)^T kappa_{n+1} and I_{n+1}'s
// dependence on h(x_n) enter the x_n equation (the parts through lambda_n
// land in the matrix, the rest in the right-hand side), the step matrix
// gets what the Newton matrix leaves out of dI_n/dx_n, and
//   dL/dp += kappa_n dG_n/dp + beta_n ag0_n q_n dc_n/dp
// (W, L through the oxide and overlap capacitances, VTO through von) with
// dh/dx and dh/dVTO from m1_meyer_dual.
#include "mos1_charge_adjoint.cuh"
#include "newton_common.cuh"
#include "tran_device.cuh"

#include <cuda_runtime.h>

namespace nsg {

// Per instance: the replayed schedule and the adjoint workspace.
struct AdjDesc {
    int32_t n_steps;     // accepted steps after t = 0
    int32_t every;       // checkpoint interval K
    int32_t probe;       // unknown in the loss
    int32_t n_ckpt;      // checkpoints (steps 0, K, 2K, ...)
    int64_t rec_off;     // first StepRecord / time / target (t = 0) of the instance
    int64_t x0_off;      // the recorded operating point
    int64_t ws_off;      // adjoint workspace
    int64_t ckpt_len;    // doubles per checkpoint
};

namespace {

// -lambda^T dF/dp of resistors, DC sources and MOSFET channels at x (the
// dc_adjoint_kernel contraction), accumulated into g.  A DC source's value
// enters every step's branch (or node) equation and the operating point,
// which the replay re-solves with the replayed parameters.
__device__ inline void grad_contract(const Inst& v, const DcDesc& d, const int32_t* prog,
                                     const double* lam, const double* x, double* g) {
    const int32_t* gp = prog + d.prog_off[DP_grad];
    auto at = [&](const double* vec, int32_t i) { return i >= 0 ? vec[i] : 0.0; };
    for (int32_t r = threadIdx.x; r < d.n_grad; r += blockDim.x) {
        const int32_t* e = gp + 5 * r;
        const int32_t kind = e[0], p = e[1], a = e[2], b = e[3];
        if (kind == 1) {
            const double R = v.par[p];
            g[p] += (at(lam, a) - at(lam, b)) * (at(x, a) - at(x, b)) / (R * R);
        } else if (kind == 2) {  // voltage source: F_branch = vp - vn - V
            g[p] += at(lam, a);
        } else if (kind == 3) {  // current source p -> n: F_p += I, F_n -= I
            g[p] += -(at(lam, a) - at(lam, b));
        } else if (kind == 4) {
            const double* P = v.par + p;
            const double* rec = v.mrec + kMosRecCount * e[4];
            const double dm = rec[kRMode];
            const double type = P[kMType];
            const double cdrain = dm * (rec[kRCd] + rec[kRCbd]);
            const double leff = P[kML] - 2 * P[kMLatDiff];
            const double dl = at(lam, a) - at(lam, b);
            g[p + kMW] += -dl * type * dm * cdrain / P[kMW];
            g[p + kML] += dl * type * dm * cdrain / leff;
            g[p + kMVto] += dl * dm * rec[kRGm];
        }
    }
}

// dq/dv of diode k's charge at junction voltage vd (DIOload's capd, without
// limiting: vd is the voltage its last load used).
__device__ inline double diode_capd(const Inst& v, int32_t k, double vd, double gmin) {
    const int32_t* dr = v.diodes + 4 * k;
    const DiodeDC r =
        diode_eval(vd, false, vd, v.dconst[3 * k], v.dconst[3 * k + 1], v.dconst[3 * k + 2], gmin,
                   diode_brk(v.par + dr[2], v.par[dr[2] + kDpVt]));
    double q, capd;
    diode_charge(v.par + dr[2], r.vd, r.cdb, r.gdb, &q, &capd);
    return capd;
}

// Integrator context of accepted step n (1-based) from its record.
__device__ inline IntegCtx step_ctx(const StepRecord& r, double t, int mode) {
    IntegCtx c{};
    for (int q = 0; q < 3; ++q) c.ag[q] = r.ag[q];
    c.xmu_ratio = r.xmu_ratio;
    c.delta = (r.ag[0] != 0.0) ? 1.0 / r.ag[0] : 0.0;
    c.delta_old[0] = c.delta;
    c.delta_old[1] = c.delta;
    c.delta_old[2] = c.delta;
    c.time = t;
    c.mode = mode;
    c.order = r.order;
    c.method = r.method;
    return c;
}

__device__ inline void vcopy(double* dst, const double* src, int64_t n) {
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

// Node voltages d, g, s, b of MOSFET record mr in x (0 for ground).
__device__ inline void mos_volts(const int32_t* mr, const double* x, double vn[4]) {
    for (int q = 0; q < 4; ++q) vn[q] = mr[q] >= 0 ? x[mr[q]] : 0.0;
}

__device__ inline bool mos_charged(const Inst& v, const int32_t* mr) {
    return mr[6] != kMosFamilyBsim4 && m1_has_charge(v.par + mr[4]);
}

__device__ inline void meyer_at(const double* P, const double vn[4], Dual4 h[3]) {
    const double type = P[kMType];
    m1_meyer_dual(P, type * (vn[1] - vn[2]), type * (vn[0] - vn[2]), type * (vn[3] - vn[2]), h);
}

// The MOSFET stamp terms of the instance's term vector.
__device__ inline double* mos_terms(const Inst& v) {
    return v.tv + v.n_const + kDiodeTermCount * v.n_diodes + kCapTermCount * v.n_caps +
           kSrcTermCount * v.n_srcs;
}

// Step n's Jacobian.  A Meyer unit's current in the step residual is
// I_n = i_n + ag0 q_n (1 - c_n): the charge integration MOS1load calls
// returns ceq = i - geq q (mos1_shim.cpp's NIintegrate) and the load adds
// ag0 q back.  Its exact derivative is
//   ag0 (2 - c_n) B dq_n/dx_n - ag0 q_n B dh(x_n)/dx
// with dq_n/dx_n = c_n B^T + (v_n - v_{n-1}) dh(x_n)/dx; the Newton matrix
// holds ag0 c_n B B^T of it, this adds the rest.
__device__ __noinline__ void meyer_jacobian(const Inst& v, const double* xs, const double* xp,
                                            double ag0) {
    double* tv_m = mos_terms(v);
    for (int32_t k = threadIdx.x; k < v.n_mos; k += blockDim.x) {
        const int32_t* mr = v.mos + kMosTabStride * k;
        if (!mos_charged(v, mr)) continue;
        const double* P = v.par + mr[4];
        const double* st0 = v.st[0] + mr[5];
        const double* st1 = v.st[1] + mr[5];
        const double type = P[kMType];
        double vn[4], vp[4];
        mos_volts(mr, xs, vn);
        mos_volts(mr, xp, vp);
        Dual4 h[3];
        meyer_at(P, vn, h);
        double* t = tv_m + kMosTermCount * k;
        for (int j = 0; j < 3; ++j) {
            const int a = m1_unit_pos(j), b = m1_unit_neg(j);
            const int slot = m1_unit_cap_slot(j);
            double dW, dL;
            const double c = st0[slot] + st1[slot] + m1_overlap(P, j, &dW, &dL);
            const double q = type * st0[slot + 1];
            const double dv = (vn[a] - vn[b]) - (vp[a] - vp[b]);
            const double gh = ag0 * ((2.0 - c) * dv - q);
            const double gb = ag0 * c * (1.0 - c);
            double gn[4];
            m1_node_grad(h[j], type, gn);
            for (int r = 0; r < 4; ++r) {
                t[m1_term_at(a, r)] += gh * gn[r];
                t[m1_term_at(b, r)] -= gh * gn[r];
            }
            t[m1_term_at(a, a)] += gb;
            t[m1_term_at(a, b)] -= gb;
            t[m1_term_at(b, a)] -= gb;
            t[m1_term_at(b, b)] += gb;
        }
    }
}

// Integration coefficients the backward recursion of step n reads: its own
// ag0 and the next steps' ag1 / ag2 / trapezoidal ratio.
struct AdjCoef {
    double ag0, ag1n, ag2n, r1;
    bool has1, has2, op;  // op: the operating point (q_0 = v_0 (2 h_0 + o), no ag0 term)
};

// MOSFET charges' part of step n's adjoint right-hand side:
//   (dG_n/dx_n)^T (ag0 mu + K) + (dG_{n+1}/dx_n)^T kappa_{n+1}
//   + beta_{n+1} ag0_{n+1} q_{n+1} dh(x_n)/dx
// per Meyer unit (K = ag1 eta_{n+1} + ag2 eta_{n+2} + kappa_{n+1}; the last
// term is step n+1's I_{n+1} through c_{n+1}'s h(x_n), beta = B^T lambda,
// kept in p1), and dq/dv B (ag0 mu + ag1 eta_{n+1} + ag2 eta_{n+2}) per
// junction.  Writes mu.
__device__ __noinline__ void mos_charge_rhs(const Inst& v, int32_t base, const double* xs,
                                            const double* xp, const AdjCoef& cf,
                                            const double* eta1, const double* eta2, double* mu,
                                            const double* kap1, const double* c1,
                                            const double* w1, const double* p1, double* lam) {
    for (int32_t k = threadIdx.x; k < v.n_mos; k += blockDim.x) {
        const int32_t* mr = v.mos + kMosTabStride * k;
        if (!mos_charged(v, mr)) continue;
        const double* P = v.par + mr[4];
        const double* st0 = v.st[0] + mr[5];
        const double* st1 = v.st[1] + mr[5];
        double vn[4], vp[4];
        mos_volts(mr, xs, vn);
        if (!cf.op) mos_volts(mr, xp, vp);
        Dual4 h[3];
        meyer_at(P, vn, h);
        for (int j = 0; j < kMos1ChargeUnits; ++j) {
            const int32_t u = base + kMos1ChargeUnits * k + j;
            const int a = m1_unit_pos(j), b = m1_unit_neg(j);
            const double m = (cf.has1 && !cf.op) ? -cf.r1 * eta1[u] : 0.0;
            if (!cf.op) mu[u] = m;
            double kj = 0.0;
            if (cf.has1) kj += cf.ag1n * eta1[u];
            if (cf.has2) kj += cf.ag2n * eta2[u];
            const double z0 = cf.op ? 0.0 : cf.ag0 * m;
            double cb;
            if (j < 3) {
                const int slot = m1_unit_cap_slot(j);
                double dW, dL;
                const double o = m1_overlap(P, j, &dW, &dL);
                const double vs = vn[a] - vn[b];
                const double c = cf.op ? 2 * st0[slot] + o : st0[slot] + st1[slot] + o;
                const double self = cf.op ? 2 * vs : vs - (vp[a] - vp[b]);
                const double z = z0 + kj + kap1[u];
                cb = z * c - kap1[u] * c1[u];
                const double ch = z * self + kap1[u] * (w1[u] - vs) + p1[u];
                double gn[4];
                m1_node_grad(h[j], P[kMType], gn);
                for (int q = 0; q < 4; ++q)
                    if (mr[q] >= 0) atomicAdd(lam + mr[q], ch * gn[q]);
            } else {
                double q, capj;
                m1_bulk_charge(P, st0[j == 3 ? kSVbd : kSVbs], j == 3, &q, &capj);
                cb = capj * (z0 + kj);
            }
            if (mr[a] >= 0) atomicAdd(lam + mr[a], cb);
            if (mr[b] >= 0) atomicAdd(lam + mr[b], -cb);
        }
    }
}

// After step n's transposed solve, per Meyer unit with beta_n = B^T lambda_n:
//   eta_n   = mu_n - beta_n
//   kappa_n = ag0 eta_n + K - ag0 (1 - c_n) beta_n
// (the last term from I_n's ag0 q_n (1 - c_n)), and
//   dL/dp  += (kappa_n dv_n + beta_n ag0 q_n) (dh(x_n)/dp + do/dp)
//           + (kappa_{n+1} dv_{n+1} + beta_{n+1} ag0_{n+1} q_{n+1}) dh(x_n)/dp
// (dv_n = v_n - v_{n-1}; the second line is c_{n+1}'s h(x_n) part).  At
// the operating point (q_0 = v_0 (2 h_0 + o), no current in R_0) kappa_0 = K
// and only the gradients.  Junction units: eta only.
__device__ __noinline__ void mos_charge_update(const Inst& v, int32_t base, const double* xs,
                                               const double* xp, const AdjCoef& cf,
                                               const double* lam, double* eta1, double* eta2,
                                               const double* mu, double* kap1, double* c1,
                                               double* w1, double* p1, double* g) {
    for (int32_t k = threadIdx.x; k < v.n_mos; k += blockDim.x) {
        const int32_t* mr = v.mos + kMosTabStride * k;
        if (!mos_charged(v, mr)) continue;
        const double* P = v.par + mr[4];
        const double* st0 = v.st[0] + mr[5];
        const double* st1 = v.st[1] + mr[5];
        const double type = P[kMType];
        double vn[4], vp[4];
        mos_volts(mr, xs, vn);
        if (!cf.op) mos_volts(mr, xp, vp);
        Dual4 h[3];
        meyer_at(P, vn, h);
        const double W = P[kMW], leff = P[kML] - 2 * P[kMLatDiff];
        double gW = 0.0, gL = 0.0, gV = 0.0;
        for (int j = 0; j < kMos1ChargeUnits; ++j) {
            const int32_t u = base + kMos1ChargeUnits * k + j;
            const int a = m1_unit_pos(j), b = m1_unit_neg(j);
            auto at = [&](int32_t i) { return i >= 0 ? lam[i] : 0.0; };
            const double beta = cf.op ? 0.0 : at(mr[a]) - at(mr[b]);
            const double e = cf.op ? 0.0 : mu[u] - beta;
            if (j < 3) {
                const int slot = m1_unit_cap_slot(j);
                double dW, dL;
                const double o = m1_overlap(P, j, &dW, &dL);
                const double c = st0[slot] + st1[slot] + o;
                const double q = type * st0[slot + 1];
                double kj = 0.0;
                if (cf.has1) kj += cf.ag1n * eta1[u];
                if (cf.has2) kj += cf.ag2n * eta2[u];
                const double kap =
                    cf.op ? kj + kap1[u] : cf.ag0 * e + kj + kap1[u] - cf.ag0 * (1.0 - c) * beta;
                const double vs = vn[a] - vn[b];
                const double own =
                    cf.op ? kap * vs : kap * (vs - (vp[a] - vp[b])) + beta * cf.ag0 * q;
                const double hf = cf.op ? 2.0 : 1.0;
                const double nxt = kap1[u] * (w1[u] - vs) + p1[u];
                const double hv = h[j].v;
                gW += own * (hf * hv / W + dW) + nxt * hv / W;
                gL += own * (hf * hv / leff + dL) + nxt * hv / leff;
                gV += own * hf * h[j].d[3] + nxt * h[j].d[3];
                if (!cf.op) {
                    c1[u] = c;
                    w1[u] = vs;
                    kap1[u] = kap;
                    p1[u] = beta * cf.ag0 * q;
                }
            }
            if (!cf.op) {
                eta2[u] = eta1[u];
                eta1[u] = e;
            }
        }
        g[mr[4] + kMW] += gW;
        g[mr[4] + kML] += gL;
        g[mr[4] + kMVto] += gV;
    }
}

}  // namespace

__global__ void __launch_bounds__(kFlowThreads, 2)
tran_adjoint_kernel(const PlanDesc* __restrict__ plans, const int32_t* __restrict__ lu_pool,
                    const DcDesc* __restrict__ descs, const TranDesc* __restrict__ tdescs,
                    const AdjDesc* __restrict__ adescs, const int32_t* __restrict__ prog,
                    const double* __restrict__ params_dc, const double* __restrict__ params_tran,
                    double* __restrict__ work, double* __restrict__ adj_ws,
                    const StepRecord* __restrict__ recs, const double* __restrict__ times,
                    const double* __restrict__ rec_x0, const double* __restrict__ targets,
                    double weight, double* __restrict__ grads, double* __restrict__ loss,
                    int32_t* __restrict__ status, NewtonOptions opt, int max_iter, int colbuf,
                    int scratch_doubles) {
    extern __shared__ double smem[];
    const DcDesc d = descs[blockIdx.x];
    const TranDesc td = tdescs[blockIdx.x];
    const AdjDesc ad = adescs[blockIdx.x];
    const PlanDesc& dpd = plans[d.plan];
    const PlanDesc& tpd = plans[td.tran_plan];
    Inst v = make_inst(d, prog, params_tran, work);
    const int32_t n = v.n, ns = d.n_states;
    const int64_t K = ad.every;
    const StepRecord* rec = recs + ad.rec_off;  // rec[s] for step s >= 1
    const double* tm = times + ad.rec_off;
    const double* tg = targets + ad.rec_off;
    double* g = grads + d.param_off;
    double* ws = adj_ws + ad.ws_off;
    // workspace: checkpoints | segment x (K+2) | segment states (K+2) |
    // eta1 | eta2 | mu | kap1 | cap1 | w1 | p1 | lam
    double* ckpt = ws;
    double* seg_x = ckpt + ad.n_ckpt * ad.ckpt_len;
    double* seg_s = seg_x + (K + 2) * n;
    // charge units: capacitors 0 .. n_caps-1, then diodes, then five per
    // MOSFET (kappa, c and v of the next step for the Meyer units)
    const int32_t mos_base = v.n_caps + v.n_diodes;
    const int32_t nq = mos_base + kMos1ChargeUnits * v.n_mos;
    double* eta1 = seg_s + (K + 2) * ns;
    double* eta2 = eta1 + nq;
    double* mu = eta2 + nq;
    double* kap1 = mu + nq;
    double* cap1 = kap1 + nq;
    double* w1 = cap1 + nq;
    double* p1 = w1 + nq;
    double* lam = p1 + nq;
    double* w = work + d.w_off;
    __shared__ IntegCtx ctx;
    __shared__ SolverState solver;
    __shared__ int32_t s_fail, s_dev_conv;
    __shared__ double s_loss;

    auto save_ckpt = [&](int64_t c, const double* xc, const double* xprev) {
        double* r = ckpt + c * ad.ckpt_len;
        vcopy(r, xc, n);
        vcopy(r + n, xprev, n);
        vcopy(r + 2 * n, v.st[1], ns);
        vcopy(r + 2 * n + ns, v.st[2], ns);
        vcopy(r + 2 * n + 2 * ns, v.mrec, kMosRecCount * v.n_mos);
    };
    // Accepted step s from the current state: Newton, then rotate the ring
    // (state3 <- state2 <- state1 <- state0).  False if Newton failed.
    auto step = [&](int64_t s) -> bool {
        if (threadIdx.x == 0) {
            ctx = step_ctx(rec[s], tm[s], kModeTran | (s == 1 ? kModeInitTran : kModeInitPred));
            solver.factored = 1;
        }
        __syncthreads();
        const NewtonOutcome r = newton(v, tpd, lu_pool, &ctx, opt, max_iter, &solver, smem, colbuf,
                                       -1, -1, 1, false, scratch_doubles, true);
        if (r.code != kDcConverged) return false;
        vcopy(v.st[3], v.st[2], ns);
        __syncthreads();
        vcopy(v.st[2], v.st[1], ns);
        __syncthreads();
        vcopy(v.st[1], v.st[0], ns);
        __syncthreads();
        return true;
    };
    auto fail_with = [&](int32_t code) {
        if (threadIdx.x == 0) status[d.index] = code;
    };
    auto dl = [&](const double* x, int64_t s) {
        return 2.0 * weight * (x[ad.probe] - tg[s]);
    };

    // ---- 1. operating point: re-solved with the replayed parameters by
    // Newton from the recorded x_0 (the DC plan's pivots); states seeded
    // from it
    v.par = params_dc + d.param_off;
    load_constants(v, opt.gmin);
    vcopy(v.x, rec_x0 + td.x0_off, n);
    vcopy(v.xold, rec_x0 + td.x0_off, n);
    for (int32_t i = threadIdx.x; i < kMosRecCount * v.n_mos; i += blockDim.x) v.mrec[i] = 0.0;
    for (int32_t i = threadIdx.x; i < 4 * ns; i += blockDim.x) v.st[0][i] = 0.0;
    if (threadIdx.x == 0) {
        ctx = IntegCtx{};
        ctx.mode = kModeTranOp | kModeInitFloat;
        ctx.order = 1;
        solver.factored = 1;
        s_dev_conv = 1;
        s_fail = 0;
        s_loss = 0.0;
    }
    __syncthreads();
    {
        const NewtonOutcome r0 = newton(v, dpd, lu_pool, &ctx, opt, max_iter, &solver, smem,
                                        colbuf, -1, -1, 1, false, scratch_doubles, true);
        if (r0.code != kDcConverged) {
            fail_with(kTranDcFailed);
            return;
        }
        vcopy(v.xold, v.x, n);
        if (threadIdx.x == 0) {
            ctx.mode = kModeTranOp | kModeInitFloat;
            s_dev_conv = 1;
        }
        __syncthreads();
    }
    // states at x_0 (q = C v_0; MOSFET voltages, twice so that the second
    // load's limiting starts from x_0's own voltages)
    for (int pass = 0; pass < 2; ++pass) {
        eval_devices(v, ctx, opt, &s_dev_conv);
        __syncthreads();
    }
    for (int32_t i = threadIdx.x; i < ns; i += blockDim.x)
        v.st[1][i] = v.st[2][i] = v.st[3][i] = v.st[0][i];
    for (int32_t i = threadIdx.x; i < d.n_grad; i += blockDim.x) {
        const int32_t* e = prog + d.prog_off[DP_grad] + 5 * i;
        g[e[1]] = 0.0;
        if (e[0] == 4) g[e[1] + kMW] = g[e[1] + kML] = g[e[1] + kMVto] = 0.0;
    }
    for (int32_t k = threadIdx.x; k < v.n_caps; k += blockDim.x) g[v.caps[5 * k + 2]] = 0.0;
    __syncthreads();
    if (threadIdx.x == 0) {
        const double e0 = v.x[ad.probe] - tg[0];
        s_loss = weight * e0 * e0;
    }
    save_ckpt(0, v.x, v.x);
    __syncthreads();

    // ---- 2. forward replay with checkpoints every K steps
    v.par = params_tran + d.param_off;
    load_constants(v, opt.gmin);
    double* xprev = seg_x;  // x_{s-1} while replaying
    vcopy(xprev, v.x, n);
    __syncthreads();
    for (int64_t s = 1; s <= ad.n_steps; ++s) {
        if (!step(s)) {
            fail_with(kTranNewtonFailed);
            return;
        }
        if (threadIdx.x == 0) {
            const double e = v.x[ad.probe] - tg[s];
            s_loss += weight * e * e;
        }
        if (s % K == 0) save_ckpt(s / K, v.x, xprev);
        __syncthreads();
        vcopy(xprev, v.x, n);
        __syncthreads();
    }
    if (threadIdx.x == 0) loss[d.index] = s_loss;

    // ---- 3. backward, segment by segment
    for (int32_t k = threadIdx.x; k < nq; k += blockDim.x)
        eta1[k] = eta2[k] = kap1[k] = cap1[k] = w1[k] = p1[k] = 0.0;
    __syncthreads();
    for (int64_t c0 = ((ad.n_steps - 1) / K) * K; c0 >= 0; c0 -= K) {
        const int64_t c1 = (c0 + K < ad.n_steps) ? c0 + K : ad.n_steps;
        // restore checkpoint c0 and re-solve steps c0+1..c1 (slot j holds step c0-1+j)
        const double* r = ckpt + (c0 / K) * ad.ckpt_len;
        vcopy(v.x, r, n);
        vcopy(seg_x + n, r, n);
        vcopy(seg_x, r + n, n);
        vcopy(v.st[0], r + 2 * n, ns);
        vcopy(v.st[1], r + 2 * n, ns);
        vcopy(seg_s + ns, r + 2 * n, ns);
        vcopy(v.st[2], r + 2 * n + ns, ns);
        vcopy(seg_s, r + 2 * n + ns, ns);
        vcopy(v.mrec, r + 2 * n + 2 * ns, kMosRecCount * v.n_mos);
        __syncthreads();
        for (int64_t s = c0 + 1; s <= c1; ++s) {
            if (!step(s)) {
                fail_with(kTranNewtonFailed);
                return;
            }
            vcopy(seg_x + (s - c0 + 1) * n, v.x, n);
            vcopy(seg_s + (s - c0 + 1) * ns, v.st[1], ns);
            __syncthreads();
        }
        for (int64_t s = c1; s > c0; --s) {
            const double* xs = seg_x + (s - c0 + 1) * n;
            const double* x1 = seg_x + (s - c0) * n;
            const double* x2 = seg_x + (s - c0 - 1) * n;
            // the Newton matrix at x_s
            vcopy(v.xold, xs, n);
            vcopy(v.st[0], seg_s + (s - c0 + 1) * ns, ns);
            vcopy(v.st[1], seg_s + (s - c0) * ns, ns);
            vcopy(v.st[2], seg_s + (s - c0 - 1) * ns, ns);
            if (threadIdx.x == 0) {
                ctx = step_ctx(rec[s], tm[s], kModeTran | kModeInitFloat);
                s_dev_conv = 1;
            }
            __syncthreads();
            eval_devices(v, ctx, opt, &s_dev_conv);
            __syncthreads();
            if (v.n_mos > 0) {
                meyer_jacobian(v, xs, x1, rec[s].ag[0]);
                __syncthreads();
            }
            assemble(v);
            const RefactorResult fr = cta_refactor_flow(tpd, lu_pool, v.a, v.lu, opt.diag_gmin,
                                                        kCheckNone, 1e-3, smem, colbuf,
                                                        v.lrows, v.urows);
            if (fr.code != kStatusOk) {
                fail_with(fr.code);
                return;
            }
            // right-hand side
            for (int32_t i = threadIdx.x; i < n; i += blockDim.x) lam[i] = 0.0;
            __syncthreads();
            if (threadIdx.x == 0) lam[ad.probe] = dl(xs, s);
            __syncthreads();
            const bool has1 = s + 1 <= ad.n_steps, has2 = s + 2 <= ad.n_steps;
            for (int32_t k = threadIdx.x; k < v.n_caps; k += blockDim.x) {
                const int32_t* cr = v.caps + 5 * k;
                const double C = v.par[cr[2]];
                const double m = has1 ? -rec[s + 1].xmu_ratio * eta1[k] : 0.0;
                mu[k] = m;
                double cc = rec[s].ag[0] * C * m;
                if (has1) cc += rec[s + 1].ag[1] * C * eta1[k];
                if (has2) cc += rec[s + 2].ag[2] * C * eta2[k];
                if (cr[0] >= 0) atomicAdd(lam + cr[0], cc);
                if (cr[1] >= 0) atomicAdd(lam + cr[1], -cc);
            }
            for (int32_t k = threadIdx.x; k < v.n_diodes; k += blockDim.x) {
                const int32_t* dr = v.diodes + 4 * k;
                const int32_t u = v.n_caps + k;
                const double capd = diode_capd(v, k, v.st[0][dr[3] + kDsV], opt.gmin);
                const double m = has1 ? -rec[s + 1].xmu_ratio * eta1[u] : 0.0;
                mu[u] = m;
                double cc = rec[s].ag[0] * capd * m;
                if (has1) cc += rec[s + 1].ag[1] * capd * eta1[u];
                if (has2) cc += rec[s + 2].ag[2] * capd * eta2[u];
                if (dr[0] >= 0) atomicAdd(lam + dr[0], cc);
                if (dr[1] >= 0) atomicAdd(lam + dr[1], -cc);
            }
            AdjCoef cf{rec[s].ag[0], has1 ? rec[s + 1].ag[1] : 0.0, has2 ? rec[s + 2].ag[2] : 0.0,
                       has1 ? rec[s + 1].xmu_ratio : 0.0, has1, has2, false};
            if (v.n_mos > 0)
                mos_charge_rhs(v, mos_base, xs, x1, cf, eta1, eta2, mu, kap1, cap1, w1, p1, lam);
            __syncthreads();
            cta_solve_transposed(tpd, lu_pool, v.lu, lam, w);
            // capacitor adjoints and dL/dC
            for (int32_t k = threadIdx.x; k < v.n_caps; k += blockDim.x) {
                const int32_t* cr = v.caps + 5 * k;
                auto at = [&](const double* vec, int32_t i) { return i >= 0 ? vec[i] : 0.0; };
                const double e = mu[k] - (at(lam, cr[0]) - at(lam, cr[1]));
                const double dv0 = at(xs, cr[0]) - at(xs, cr[1]);
                const double dv1 = at(x1, cr[0]) - at(x1, cr[1]);
                const double dv2 = at(x2, cr[0]) - at(x2, cr[1]);
                g[cr[2]] += e * (rec[s].ag[0] * dv0 + rec[s].ag[1] * dv1 + rec[s].ag[2] * dv2);
                eta2[k] = eta1[k];
                eta1[k] = e;
            }
            for (int32_t k = threadIdx.x; k < v.n_diodes; k += blockDim.x) {
                const int32_t* dr = v.diodes + 4 * k;
                const int32_t u = v.n_caps + k;
                auto at = [&](const double* vec, int32_t i) { return i >= 0 ? vec[i] : 0.0; };
                const double e = mu[u] - (at(lam, dr[0]) - at(lam, dr[1]));
                eta2[u] = eta1[u];
                eta1[u] = e;
            }
            if (v.n_mos > 0) {
                mos_charge_update(v, mos_base, xs, x1, cf, lam, eta1, eta2, mu, kap1, cap1, w1, p1,
                                  g);
                __syncthreads();
            }
            grad_contract(v, d, prog, lam, xs, g);
            __syncthreads();
        }
    }

    // ---- 4. the operating point: DC Jacobian, cotangent from steps 1 and 2
    const double* x0 = ckpt;  // checkpoint 0 holds the re-solved x_0
    v.par = params_dc + d.param_off;
    load_constants(v, opt.gmin);
    vcopy(v.xold, x0, n);
    const double* r0 = ckpt;
    vcopy(v.mrec, r0 + 2 * n + 2 * ns, kMosRecCount * v.n_mos);
    vcopy(v.st[0], r0 + 2 * n, ns);
    if (threadIdx.x == 0) {
        ctx = IntegCtx{};
        ctx.mode = kModeTranOp | kModeInitFloat;
        ctx.order = 1;
        s_dev_conv = 1;
    }
    __syncthreads();
    eval_devices(v, ctx, opt, &s_dev_conv);
    __syncthreads();
    assemble(v);
    const RefactorResult fr = cta_refactor_flow(dpd, lu_pool, v.a, v.lu, opt.diag_gmin, kCheckNone,
                                                1e-3, smem, colbuf, v.lrows, v.urows);
    if (fr.code != kStatusOk) {
        fail_with(fr.code);
        return;
    }
    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) lam[i] = 0.0;
    __syncthreads();
    if (threadIdx.x == 0) lam[ad.probe] = dl(x0, 0);
    __syncthreads();
    for (int32_t k = threadIdx.x; k < v.n_caps; k += blockDim.x) {
        const int32_t* cr = v.caps + 5 * k;
        const double C = v.par[cr[2]];
        double cc = 0.0;
        if (ad.n_steps >= 1) cc += rec[1].ag[1] * C * eta1[k];
        if (ad.n_steps >= 2) cc += rec[2].ag[2] * C * eta2[k];
        if (cr[0] >= 0) atomicAdd(lam + cr[0], cc);
        if (cr[1] >= 0) atomicAdd(lam + cr[1], -cc);
    }
    for (int32_t k = threadIdx.x; k < v.n_diodes; k += blockDim.x) {
        const int32_t* dr = v.diodes + 4 * k;
        const int32_t u = v.n_caps + k;
        auto at = [&](const double* vec, int32_t i) { return i >= 0 ? vec[i] : 0.0; };
        const double capd = diode_capd(v, k, at(x0, dr[0]) - at(x0, dr[1]), opt.gmin);
        double cc = 0.0;
        if (ad.n_steps >= 1) cc += rec[1].ag[1] * capd * eta1[u];
        if (ad.n_steps >= 2) cc += rec[2].ag[2] * capd * eta2[u];
        if (dr[0] >= 0) atomicAdd(lam + dr[0], cc);
        if (dr[1] >= 0) atomicAdd(lam + dr[1], -cc);
    }
    const AdjCoef cf0{0.0, ad.n_steps >= 1 ? rec[1].ag[1] : 0.0,
                      ad.n_steps >= 2 ? rec[2].ag[2] : 0.0, 0.0, ad.n_steps >= 1,
                      ad.n_steps >= 2, true};
    if (v.n_mos > 0)
        mos_charge_rhs(v, mos_base, x0, x0, cf0, eta1, eta2, mu, kap1, cap1, w1, p1, lam);
    __syncthreads();
    cta_solve_transposed(dpd, lu_pool, v.lu, lam, w);
    if (v.n_mos > 0) {
        mos_charge_update(v, mos_base, x0, x0, cf0, lam, eta1, eta2, mu, kap1, cap1, w1, p1,
                          g);
        __syncthreads();
    }
    grad_contract(v, d, prog, lam, x0, g);
    __syncthreads();
    if (threadIdx.x == 0) status[d.index] = kStatusOk;
}

cudaError_t launch_tran_adjoint(const PlanDesc* plans, const int32_t* lu_pool, const DcDesc* descs,
                                const TranDesc* tdescs, const AdjDesc* adescs, int count,
                                const int32_t* prog, const double* params_dc,
                                const double* params_tran, double* work, double* adj_ws,
                                const StepRecord* recs, const double* times, const double* rec_x0,
                                const double* targets, double weight, double* grads, double* loss,
                                int32_t* status, const NewtonOptions& opt, int max_iter,
                                int max_col, int max_n, cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    const int colbuf = (max_col + 31) & ~31;
    const size_t a = flow_smem_bytes(colbuf, max_n), b = flow_solve_smem_bytes(max_n);
    const size_t smem = ((a > b ? a : b) + 15) & ~size_t{15};
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(tran_adjoint_kernel,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             200 * 1024);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    tran_adjoint_kernel<<<count, kFlowThreads, smem, stream>>>(
        plans, lu_pool, descs, tdescs, adescs, prog, params_dc, params_tran, work, adj_ws, recs,
        times, rec_x0, targets, weight, grads, loss, status, opt, max_iter, colbuf,
        static_cast<int>(smem / sizeof(double)));
    return cudaGetLastError();
}

}  // namespace nsg
