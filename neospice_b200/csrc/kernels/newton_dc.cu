// Batched DC operating point: the whole Newton loop of newton_solve
// (src/core/newton.cpp:51-419) for one circuit instance per CTA, in a single
// launch for the batch.  Each iteration: device loads (diodes), matrix and
// right-hand-side assembly from the stamp program, fixed-pivot refactor
// (dataflow), forward/backward solve, the NIiter convergence test and the
// INITJCT -> INITFIX -> INITFLOAT mode cascade.  Instances converge and stop
// independently (per-instance convergence mask = its CTA leaving the loop).
#include "dc_device.cuh"
#include "diode_model.cuh"
#include "lu_cta.cuh"

#include <cuda_runtime.h>

namespace nsg {

namespace {

constexpr int kModeInitFloat = 0x100;  // CKTmode bits (newton.cpp:109-115)
constexpr int kModeInitJct = 0x200;
constexpr int kModeInitFix = 0x400;

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

}  // namespace

// Two CTAs per SM: registers are capped at 64 per thread.
__global__ void __launch_bounds__(kFlowThreads, 2)
newton_dc_kernel(const PlanDesc* __restrict__ plans, const int32_t* __restrict__ lu_pool,
                 const DcDesc* __restrict__ descs, const int32_t* __restrict__ prog,
                 const double* __restrict__ params, double* __restrict__ work,
                 double* __restrict__ solutions, int32_t* __restrict__ status,
                 int32_t* __restrict__ iterations, NewtonOptions opt, int colbuf) {
    extern __shared__ double smem[];
    const DcDesc d = descs[blockIdx.x];
    const PlanDesc& pd = plans[d.plan];
    const int32_t n = d.n;
    const int32_t* slot_ptr = prog + d.prog_off[DP_slot_ptr];
    const int32_t* slot_terms = prog + d.prog_off[DP_slot_terms];
    const int32_t* rhs_ptr = prog + d.prog_off[DP_rhs_ptr];
    const int32_t* rhs_terms = prog + d.prog_off[DP_rhs_terms];
    const int32_t* ucb_ptr = prog + d.prog_off[DP_ucb_ptr];
    const int32_t* ucb_terms = prog + d.prog_off[DP_ucb_terms];
    const int32_t* term_op = prog + d.prog_off[DP_term_op];
    const int32_t* term_param = prog + d.prog_off[DP_term_param];
    const int32_t* diodes = prog + d.prog_off[DP_diodes];  // (pos, neg, param) triples
    const double* par = params + d.param_off;
    double* x = work + d.x_off;
    double* xold = work + d.xold_off;
    double* a = work + d.a_off;
    double* lu = work + d.lu_off;
    double* lrows = work + d.lrows_off;
    double* urows = work + d.urows_off;
    double* tv = work + d.tv_off;
    double* dstate = work + d.dstate_off;   // (vd, cd, gd) per diode
    double* dconst = work + d.dconst_off;   // (csat, vte, vcrit) per diode

    __shared__ int32_t s_conv, s_dev_conv;
    const double vt = kKoverQTimesTnom;

    // Prologue: constant term values, diode constants, zero initial guess.
    for (int32_t k = threadIdx.x; k < d.n_const; k += blockDim.x) {
        const int32_t pi = term_param[k];
        tv[k] = term_value(term_op[k], pi >= 0 ? par[pi] : 0.0, opt.gmin);
    }
    for (int32_t k = threadIdx.x; k < d.n_diodes; k += blockDim.x) {
        const int32_t pi = diodes[3 * k + 2];
        const double csat = par[pi];
        const double vte = par[pi + 1] * vt;
        dconst[3 * k] = csat;
        dconst[3 * k + 1] = vte;
        dconst[3 * k + 2] = diode_vcrit(vte, csat);
        dstate[3 * k] = dstate[3 * k + 1] = dstate[3 * k + 2] = 0.0;
    }
    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) x[i] = 0.0;
    __syncthreads();

    int mode = kModeInitJct;
    bool force_numeric = false;
    bool first_numeric = true;
    int32_t result = kDcNoConvergence;
    int32_t iters = opt.max_iter;

    for (int iter = 0; iter < opt.max_iter; ++iter) {
        for (int32_t i = threadIdx.x; i < n; i += blockDim.x) xold[i] = x[i];
        if (threadIdx.x == 0) s_dev_conv = 1;
        __syncthreads();

        // Device loads: diodes (DIOload), writing their dynamic terms.
        const bool initjct = (mode & kModeInitJct) != 0;
        for (int32_t k = threadIdx.x; k < d.n_diodes; k += blockDim.x) {
            const int32_t pos = diodes[3 * k], neg = diodes[3 * k + 1];
            const double vp = pos >= 0 ? xold[pos] : 0.0;
            const double vn = neg >= 0 ? xold[neg] : 0.0;
            const DiodeDC r = diode_dc_load(initjct, vp, vn, dstate[3 * k], dconst[3 * k],
                                            dconst[3 * k + 1], dconst[3 * k + 2], opt.gmin);
            dstate[3 * k] = r.vd;
            dstate[3 * k + 1] = r.cd;
            dstate[3 * k + 2] = r.gd;
            const double cdeq = r.cd - r.gd * r.vd;
            double* t = tv + d.n_const + kDiodeTermCount * k;
            t[0] = r.gd;
            t[1] = r.gd + 0.0;
            t[2] = -r.gd;
            t[3] = cdeq;
            t[4] = -cdeq;
            // DIODevice::conv_test (dio_device.cpp:296-307) on the stored state
            const double delvd = (vp - vn) - r.vd;
            const double cdhat = r.cd + r.gd * delvd;
            const double tol = opt.reltol * fmax(fabs(cdhat), fabs(r.cd)) + opt.abstol;
            const bool ok = (r.check == 0) && (fabs(cdhat - r.cd) <= tol);
            if (!ok) s_dev_conv = 0;
        }
        __syncthreads();

        // Assembly: every slot / row sums its terms in load order.
        for (int32_t s = threadIdx.x; s < d.nnz; s += blockDim.x) {
            double v = 0.0;
            for (int32_t k = slot_ptr[s]; k < slot_ptr[s + 1]; ++k) v = __dadd_rn(v, tv[slot_terms[k]]);
            a[s] = v;
        }
        for (int32_t i = threadIdx.x; i < n; i += blockDim.x) {
            double v = 0.0, u = 0.0;
            for (int32_t k = rhs_ptr[i]; k < rhs_ptr[i + 1]; ++k) v = __dadd_rn(v, tv[rhs_terms[k]]);
            for (int32_t k = ucb_ptr[i]; k < ucb_ptr[i + 1]; ++k) u = __dadd_rn(u, tv[ucb_terms[k]]);
            x[i] = __dadd_rn(v, u);
        }
        __syncthreads();

        // Factor: numeric (first iteration, or after a mode flip / singular
        // refactor) re-validates pivots; refactorize checks zero pivots only.
        const bool numeric = force_numeric || initjct;
        const RefactorResult fr = cta_refactor_flow(pd, lu_pool, a, lu, opt.diag_gmin,
                                                    numeric && !first_numeric, 1e-3, smem, colbuf,
                                                    lrows, urows);
        if (fr.code == kStatusTimeout) {
            result = kStatusTimeout;
            iters = iter + 1;
            break;
        }
        if (numeric) {
            if (fr.code != kStatusOk) {
                // NeoSolver::numeric would re-order (103) or report singular.
                result = fr.code;
                iters = iter + 1;
                break;
            }
            first_numeric = false;
            force_numeric = false;
        } else if (fr.code != kStatusOk) {
            force_numeric = true;  // newton.cpp:229-234: retry with numeric
            for (int32_t i = threadIdx.x; i < n; i += blockDim.x) x[i] = xold[i];
            __syncthreads();
            continue;
        }

        if (!cta_solve_flow(pd, lu_pool, lu, lrows, urows, x, smem)) {
            result = kStatusTimeout;
            iters = iter + 1;
            break;
        }

        // Convergence test (newton.cpp:267-292).
        if (threadIdx.x == 0) s_conv = 1;
        __syncthreads();
        for (int32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const double vn = x[i], vo = xold[i];
            bool ok = !(isnan(vn) || isinf(vn));
            if (ok) {
                const double tol = opt.reltol * fmax(fabs(vn), fabs(vo)) +
                                   (i < d.num_nodes ? opt.vntol : opt.abstol);
                ok = fabs(vn - vo) <= tol;
            }
            if (!ok) s_conv = 0;
        }
        __syncthreads();
        bool conv = (s_conv != 0) && iter > 0 && (s_dev_conv != 0);

        if (mode & kModeInitFloat) {
            if (conv) {
                result = kDcConverged;
                iters = iter + 1;
                break;  // the returned solution is the previous iterate
            }
        } else if (mode & kModeInitJct) {
            mode = kModeInitFix;
            force_numeric = true;
        } else if (mode & kModeInitFix) {
            if (conv) mode = kModeInitFloat;
        }
        __syncthreads();
    }
    __syncthreads();
    double* out = solutions + d.sol_off;
    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) out[i] = xold[i];
    if (threadIdx.x == 0) {
        status[d.index] = result;
        iterations[d.index] = iters;
    }
}

size_t dc_smem_bytes(int max_col, int max_n) {
    const int colbuf = (max_col + 31) & ~31;
    const size_t a = flow_smem_bytes(colbuf, max_n);
    const size_t b = flow_solve_smem_bytes(max_n);
    return a > b ? a : b;
}

cudaError_t launch_newton_dc(const PlanDesc* plans, const int32_t* lu_pool, const DcDesc* descs,
                             int count, const int32_t* prog, const double* params, double* work,
                             double* solutions, int32_t* status, int32_t* iterations,
                             const NewtonOptions& opt, int max_col, int max_n,
                             cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    const int colbuf = (max_col + 31) & ~31;
    const size_t smem = dc_smem_bytes(max_col, max_n);
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(newton_dc_kernel,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             200 * 1024);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    newton_dc_kernel<<<count, kFlowThreads, smem, stream>>>(plans, lu_pool, descs, prog, params,
                                                             work, solutions, status, iterations,
                                                             opt, colbuf);
    return cudaGetLastError();
}

}  // namespace nsg
