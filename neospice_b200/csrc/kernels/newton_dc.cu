// Batched DC operating point: solve_dc (src/core/dc.cpp:53-175; newton_solve,
// src/core/newton.cpp:51-419) with its direct attempt and the gmin-stepping
// aids, for one circuit instance per CTA, all instances in a single launch.
// Each iteration: device loads, matrix and right-hand-side assembly from the
// stamp program, fixed-pivot refactor (dataflow), forward/backward solve, the
// NIiter convergence test and the INITJCT -> INITFIX -> INITFLOAT cascade.
// Instances converge and stop independently (per-instance convergence mask =
// its CTA leaving the loop).
#include "dc_op.cuh"

#include <cuda_runtime.h>

namespace nsg {

// Two CTAs per SM: registers are capped at 64 per thread.  subset (optional)
// lists the descriptor positions to run, one per block.  ctls[index] is the
// instance's operating-point controller: zeroed by the host for a fresh run,
// kept across launches when an instance stopped with kStatusReorder.
__global__ void __launch_bounds__(kFlowThreads, 2)
newton_dc_kernel(const PlanDesc* __restrict__ plans, const int32_t* __restrict__ lu_pool,
                 const DcDesc* __restrict__ descs, const int32_t* __restrict__ subset,
                 const int32_t* __restrict__ prog, const double* __restrict__ params,
                 double* __restrict__ work, double* __restrict__ solutions,
                 int32_t* __restrict__ status, int32_t* __restrict__ iterations,
                 DcCtl* __restrict__ ctls, NewtonOptions opt, int colbuf, int scratch_doubles,
                 int stage_doubles, int plan_words, int32_t* rmaps, int64_t rmap_stride) {
    extern __shared__ double smem[];
    const DcDesc d = descs[subset ? subset[blockIdx.x] : blockIdx.x];
    __shared__ PlanDesc s_pd;
    const int32_t* pool = stage_plan(
        plans[d.plan], lu_pool,
        plan_words > 0 ? reinterpret_cast<int32_t*>(smem + scratch_doubles + stage_doubles) : nullptr,
        plan_words, &s_pd);
    const PlanDesc& pd = s_pd;
    double* stage = (d.stage_len <= stage_doubles) ? smem + scratch_doubles : nullptr;
    stage_copy(d, work, stage, true);
    // Per-thread views (not a shared copy as in the transient kernel): the
    // dataflow scratch of large meshes fills the shared memory of two CTAs
    // per SM to within a few hundred bytes.
    Inst v = make_inst(d, prog, params, work, stage);
    static_assert(kFlowWarps == 16, "the host sizes the row maps for 16 warps per CTA");
    if (rmaps) {
        v.rmaps = rmaps + static_cast<int64_t>(blockIdx.x) * kFlowWarps * rmap_stride;
        v.rmap_stride = rmap_stride;
    }
    __shared__ IntegCtx ctx;
    __shared__ SolverState solver;
    __shared__ int32_t s_fresh;
    DcCtl* ctl = ctls + d.index;
    constexpr int kFirst = kModeDcOp | kModeInitJct, kCont = kModeDcOp | kModeInitFloat;

    if (threadIdx.x == 0) s_fresh = (ctl->active == 0);
    __syncthreads();
    const bool fresh = s_fresh != 0;
    if (fresh) {
        for (int32_t k = threadIdx.x; k < kMosRecCount * v.n_mos; k += blockDim.x) v.mrec[k] = 0.0;
        for (int32_t k = threadIdx.x; k < 4 * d.n_states; k += blockDim.x) v.st[0][k] = 0.0;
        for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) v.x[i] = 0.0;
    }
    if (threadIdx.x == 0) {
        if (fresh) dc_op_start(ctl, kFirst, opt.first_aid);
        ctx = IntegCtx{};
        ctx.order = 1;
        ctx.time = 0.0;
        solver.factored = fresh ? 0 : 1;
    }
    __syncthreads();
    // solve_dc (dc.cpp:53-175): direct attempt, true gmin stepping, gmin stepping
    const int32_t code = dc_operating_point(v, d.n_states, pd, pool, &ctx, &solver, ctl, opt,
                                            kFirst, kCont, true, work + d.dcsave_off, smem, colbuf,
                                            scratch_doubles);

    stage_copy(d, work, stage, false);
    double* out = solutions + d.sol_off;
    for (int32_t i = threadIdx.x; i < v.n; i += blockDim.x) out[i] = v.x[i];
    if (threadIdx.x == 0) {
        status[d.index] = code;
        iterations[d.index] = ctl->total;
    }
}

size_t dc_smem_bytes(int max_col, int max_n) {
    const int colbuf = (max_col + 31) & ~31;
    const size_t a = flow_smem_bytes(colbuf, max_n);
    const size_t b = flow_solve_smem_bytes(max_n);
    return a > b ? a : b;
}

cudaError_t launch_newton_dc(const PlanDesc* plans, const int32_t* lu_pool, const DcDesc* descs,
                             const int32_t* subset, int count, const int32_t* prog,
                             const double* params, double* work, double* solutions,
                             int32_t* status, int32_t* iterations, DcCtl* ctls,
                             const NewtonOptions& opt, int max_col, int max_n,
                             long long max_stage, int32_t* rmaps, cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    const int colbuf = (max_col + 31) & ~31;
    const size_t scratch = (dc_smem_bytes(max_col, max_n) + 15) & ~size_t{15};
    const size_t plan = (max_n <= 128) ? kPlanStageBytes : 0;
    const size_t stage = stage_bytes_for(scratch + plan, max_stage);
    const size_t smem = scratch + stage + plan;
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(newton_dc_kernel,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             200 * 1024);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    newton_dc_kernel<<<count, kFlowThreads, smem, stream>>>(plans, lu_pool, descs, subset, prog,
                                                             params, work, solutions, status,
                                                             iterations, ctls, opt, colbuf,
                                                             static_cast<int>(scratch / sizeof(double)),
                                                             static_cast<int>(stage / sizeof(double)),
                                                             static_cast<int>(plan / sizeof(int32_t)),
                                                             rmaps, max_n);
    return cudaGetLastError();
}

}  // namespace nsg
