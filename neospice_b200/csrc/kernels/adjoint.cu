// Batched DC adjoint: gradients of a scalar loss L(x) through the DC
// operating point x(p) (F(x, p) = 0) with respect to the circuit parameters,
// for one instance per CTA.  With J the MNA Jacobian at the converged x:
//   J^T lambda = dL/dx,     dL/dp = -lambda^T dF/dp.
// J is re-evaluated at x (device loads in MODEDCOP | MODEINITFLOAT, the same
// fixed-pivot refactor as the forward solve), lambda comes from the
// transposed solve on those factors (SparseMatrix::solve_transposed,
// src/solver/solve.cpp:102-141), and the contraction runs over the circuit's
// gradient program: resistors, DC voltage and current sources, and the W, L
// and VTO of level-1 MOSFETs (the reference's .sens, src/core/sens.cpp:57-140,
// covers R, V and I by finite differences).
#include "newton_common.cuh"

#include <cuda_runtime.h>

namespace nsg {

__global__ void __launch_bounds__(kFlowThreads, 2)
dc_adjoint_kernel(const PlanDesc* __restrict__ plans, const int32_t* __restrict__ lu_pool,
                  const DcDesc* __restrict__ descs, const int32_t* __restrict__ prog,
                  const double* __restrict__ params, double* __restrict__ work,
                  const double* __restrict__ solutions, const double* __restrict__ cotangent,
                  double* __restrict__ grads, int32_t* __restrict__ status, NewtonOptions opt,
                  int colbuf) {
    extern __shared__ double smem[];
    const DcDesc d = descs[blockIdx.x];
    const PlanDesc& pd = plans[d.plan];
    const Inst v = make_inst(d, prog, params, work);
    __shared__ IntegCtx ctx;
    __shared__ int32_t s_dev_conv;
    const double* xs = solutions + d.sol_off;

    load_constants(v, opt.gmin);
    for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) v.xold[i] = xs[i];
    if (threadIdx.x == 0) {
        ctx = IntegCtx{};
        ctx.mode = kModeDcOp | kModeInitFloat;
        ctx.order = 1;
        s_dev_conv = 1;
    }
    __syncthreads();
    eval_devices(v, ctx, opt, &s_dev_conv);  // the Jacobian at the solution
    __syncthreads();
    assemble(v);
    const RefactorResult fr = cta_refactor_flow(pd, lu_pool, v.a, v.lu, opt.diag_gmin, 0, 1e-3,
                                                smem, colbuf, v.lrows, v.urows);
    if (fr.code != kStatusOk) {
        if (threadIdx.x == 0) status[d.index] = fr.code;
        return;
    }
    double* lam = v.x;
    for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) lam[i] = cotangent[d.sol_off + i];
    double* w = work + d.w_off;
    cta_solve_transposed(pd, lu_pool, v.lu, lam, w);

    const int32_t* gp = prog + d.prog_off[DP_grad];
    double* g = grads + d.param_off;
    auto at = [&](const double* vec, int32_t i) { return i >= 0 ? vec[i] : 0.0; };
    for (int32_t r = threadIdx.x; r < d.n_grad; r += blockDim.x) {
        const int32_t* e = gp + 5 * r;
        const int32_t kind = e[0], p = e[1], a = e[2], b = e[3];
        if (kind == 1) {          // resistor: F_a += (va - vb)/R, F_b -= (va - vb)/R
            const double R = v.par[p];
            g[p] = (at(lam, a) - at(lam, b)) * (at(xs, a) - at(xs, b)) / (R * R);
        } else if (kind == 2) {   // voltage source: F_branch = vp - vn - V
            g[p] = at(lam, a);
        } else if (kind == 3) {   // current source p -> n: F_p += I, F_n -= I
            g[p] = -(at(lam, a) - at(lam, b));
        } else if (kind == 4) {   // MOSFET channel current: F_d = type*mode*cdrain = -F_s
            const double* P = v.par + p;
            const double* rec = v.mrec + kMosRecCount * e[4];
            const double dm = rec[kRMode];
            const double type = P[kMType];
            const double cdrain = dm * (rec[kRCd] + rec[kRCbd]);
            const double leff = P[kML] - 2 * P[kMLatDiff];
            const double dl = at(lam, a) - at(lam, b);
            g[p + kMW] = -dl * type * dm * cdrain / P[kMW];
            g[p + kML] = dl * type * dm * cdrain / leff;
            g[p + kMVto] = dl * dm * rec[kRGm];
        }
    }
    if (threadIdx.x == 0) status[d.index] = kStatusOk;
}

cudaError_t launch_dc_adjoint(const PlanDesc* plans, const int32_t* lu_pool, const DcDesc* descs,
                              int count, const int32_t* prog, const double* params, double* work,
                              const double* solutions, const double* cotangent, double* grads,
                              int32_t* status, const NewtonOptions& opt, int max_col, int max_n,
                              cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    const int colbuf = (max_col + 31) & ~31;
    const size_t smem = flow_smem_bytes(colbuf, max_n);
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(dc_adjoint_kernel,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             200 * 1024);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    dc_adjoint_kernel<<<count, kFlowThreads, smem, stream>>>(plans, lu_pool, descs, prog, params,
                                                             work, solutions, cotangent, grads,
                                                             status, opt, colbuf);
    return cudaGetLastError();
}

}  // namespace nsg
