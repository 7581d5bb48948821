// Batched fixed-pivot sparse LU refactor and triangular sweeps (FP64).
//
// One CTA owns one circuit instance; instances may have different sizes,
// patterns and pivot orders (each InstDesc points at its own PlanDesc).
// Inside a CTA, columns (rows) of one level of the dependency DAG run
// concurrently, a warp per column for the refactor and a thread per row for
// the sweeps, with __syncthreads() between levels.
//
// Rounding order.  Every value is produced by the same sequence of IEEE
// double operations as the reference's SparseMatrix::factor / solve /
// solve_transposed (src/solver/factor.cpp:980-1052, solve.cpp:6-47,
// :102-141): updates into one entry are applied in ascending pivot order, one
// at a time, with separately rounded multiply and subtract (__dmul_rn,
// __dsub_rn: no FMA contraction).  Results are therefore bit-identical to the
// reference under the same pivot sequence.
#include "lu_cta.cuh"

#include <cuda_runtime.h>

namespace nsg {

namespace {
struct PlanView {
    const int32_t* a[PA_COUNT];
    __device__ PlanView(const PlanDesc& d, const int32_t* pool) {
#pragma unroll
        for (int k = 0; k < PA_COUNT; ++k) a[k] = pool + d.off[k];
    }
    __device__ const int32_t* operator[](int k) const { return a[k]; }
};
__device__ __forceinline__ double mul(double x, double y) { return __dmul_rn(x, y); }
__device__ __forceinline__ double sub(double x, double y) { return __dsub_rn(x, y); }
}  // namespace

// Load A into the LU pattern, add diag_gmin to every pivot (AMD-LU: to the
// column's own diagonal entry of A), then eliminate column by column.
// check_pivots is a kCheck* mode.  Markowitz plans: kCheckNumeric applies the
// re-validation test of SparseMatrix::order_and_factor (factor.cpp:929-947):
// the pivot must exceed rel_threshold times the largest entry below it, else
// the instance is flagged kStatusReorder at that step; otherwise only an
// exact zero pivot is flagged (kStatusSingular), as in SparseMatrix::factor.
// AMD-LU plans follow amd_column_status.
__global__ void __launch_bounds__(256)
refactor_kernel(const PlanDesc* __restrict__ plans, const int32_t* __restrict__ pool,
                const InstDesc* __restrict__ insts, const double* __restrict__ A,
                double* __restrict__ LU, double diag_gmin, int check_pivots,
                double rel_threshold, int32_t* __restrict__ status,
                int32_t* __restrict__ fail_step) {
    const InstDesc inst = insts[blockIdx.x];
    const PlanDesc& pd = plans[inst.plan];
    const PlanView p(pd, pool);
    const int32_t* col_ptr = p[PA_col_ptr];
    const int32_t* row_idx = p[PA_row_idx];
    const int32_t* diag_pos = p[PA_diag_pos];
    const int32_t* lu_src = p[PA_lu_src];
    const int32_t* upd_start = p[PA_upd_start];
    const int32_t* upd_dst = p[PA_upd_dst];
    const int32_t map16 = pd.map16;
    const int32_t* lev_ptr = p[PA_col_lev_ptr];
    const int32_t* lev = p[PA_col_lev];
    const double* a = A + inst.a_off;
    double* lu = LU + inst.lu_off;

    const bool amd = pd.kind == kPlanAmdLu;
    const int32_t* piv_rank = p[PA_piv_rank];
    const int32_t* gmin_pos = p[PA_gmin_pos];
    __shared__ unsigned long long s_fail;
    __shared__ int32_t s_growth;
    if (threadIdx.x == 0) {
        s_fail = ~0ull;
        s_growth = 0;
    }

    for (int32_t q = threadIdx.x; q < pd.nnz_lu; q += blockDim.x) {
        const int32_t s = lu_src[q];
        lu[q] = (s >= 0) ? a[s] : 0.0;
    }
    __syncthreads();
    if (diag_gmin != 0.0)
        for (int32_t j = threadIdx.x; j < pd.n; j += blockDim.x) {
            const int32_t g = amd ? (gmin_pos[j] < 0 ? -1 : col_ptr[j] + gmin_pos[j]) : diag_pos[j];
            if (g >= 0) lu[g] = __dadd_rn(lu[g], diag_gmin);
        }
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    for (int32_t l = 0; l < pd.n_col_lev; ++l) {
        for (int32_t k = lev_ptr[l] + warp; k < lev_ptr[l + 1]; k += nwarps) {
            const int32_t j = lev[k];
            const int32_t dj = diag_pos[j];
            double colmax = 0.0;
            for (int32_t q = col_ptr[j]; q < dj; ++q) {
                const int32_t r = row_idx[q];
                const double u = amd ? lu[q] : mul(lu[q], lu[diag_pos[r]]);
                colmax = fmax(colmax, fabs(u));
                __syncwarp();
                if (lane == 0) lu[q] = u;
                const int32_t l0 = diag_pos[r] + 1;
                const int32_t cnt = col_ptr[r + 1] - l0;
                const int32_t us = upd_start[q];
                const int32_t c0 = col_ptr[j];
                for (int32_t t = lane; t < cnt; t += 32) {
                    const int32_t d = c0 + upd_at(upd_dst, map16, us + t);
                    lu[d] = sub(lu[d], mul(u, lu[l0 + t]));
                }
                __syncwarp();
            }
            const double piv = lu[dj];
            const int32_t c0 = col_ptr[j];
            const int32_t len = col_ptr[j + 1] - c0;
            int32_t code;
            if (amd) {
                const AmdColumn v = amd_column_status(lu + c0, dj - c0, len, colmax, check_pivots,
                                                      piv_rank[j], gmin_pos[j], lane);
                code = v.code;
                if (lane == 0 && v.growth_fail) s_growth = 1;
            } else if (check_pivots == kCheckNumeric) {
                double largest = 0.0;
                for (int32_t q = dj + 1 + lane; q < col_ptr[j + 1]; q += 32)
                    largest = fmax(largest, fabs(lu[q]));
                largest = warp_max(largest);
                code = !(largest * rel_threshold < fabs(piv)) ? kStatusReorder : kStatusOk;
            } else {
                code = (piv == 0.0) ? kStatusSingular : kStatusOk;
            }
            __syncwarp();
            if (amd) {
                for (int32_t q = dj + 1 + lane; q < col_ptr[j + 1]; q += 32)
                    lu[q] = __ddiv_rn(lu[q], piv);
            } else if (lane == 0) {
                lu[dj] = 1.0 / piv;
            }
            if (lane == 0 && code != kStatusOk) atomicMin(&s_fail, fail_key(j, code));
            __syncwarp();
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const bool ok = s_fail == ~0ull || (amd && !amd_verdict_counts(check_pivots, s_growth != 0));
        status[inst.index] = ok ? kStatusOk : static_cast<int32_t>(s_fail & 0xffffffffu);
        if (fail_step) fail_step[inst.index] = ok ? -1 : static_cast<int32_t>(s_fail >> 32);
    }
}

// Dataflow refactor (cta_refactor_flow), one CTA per instance.
__global__ void __launch_bounds__(kFlowThreads)
refactor_flow_kernel(const PlanDesc* __restrict__ plans, const int32_t* __restrict__ pool,
                     const InstDesc* __restrict__ insts, const double* __restrict__ A,
                     double* __restrict__ LU, double diag_gmin, int check_pivots,
                     double rel_threshold, int32_t* __restrict__ status,
                     int32_t* __restrict__ fail_step, int colbuf,
                     double* __restrict__ lrows, double* __restrict__ urows) {
    extern __shared__ double smem[];
    const InstDesc inst = insts[blockIdx.x];
    const RefactorResult r =
        cta_refactor_flow(plans[inst.plan], pool, A + inst.a_off, LU + inst.lu_off, diag_gmin,
                          check_pivots, rel_threshold, smem, colbuf, lrows + inst.lrows_off,
                          urows + inst.urows_off);
    if (threadIdx.x == 0) {
        status[inst.index] = r.code;
        if (fail_step) fail_step[inst.index] = r.step;
    }
}

// x <- A^{-1} x with the factored LU (SparseMatrix::solve).
__global__ void __launch_bounds__(256)
solve_kernel(const PlanDesc* __restrict__ plans, const int32_t* __restrict__ pool,
             const InstDesc* __restrict__ insts, const double* __restrict__ LU,
             double* __restrict__ X, double* __restrict__ W) {
    const InstDesc inst = insts[blockIdx.x];
    cta_solve(plans[inst.plan], pool, LU + inst.lu_off, X + inst.x_off, W + inst.w_off);
}

// x <- A^{-1} x, dataflow sweeps on the row-major copies (cta_solve_flow).
__global__ void __launch_bounds__(kFlowThreads)
solve_flow_kernel(const PlanDesc* __restrict__ plans, const int32_t* __restrict__ pool,
                  const InstDesc* __restrict__ insts, const double* __restrict__ LU,
                  const double* __restrict__ lrows, const double* __restrict__ urows,
                  double* __restrict__ X) {
    extern __shared__ double smem[];
    const InstDesc inst = insts[blockIdx.x];
    cta_solve_flow(plans[inst.plan], pool, LU + inst.lu_off, lrows + inst.lrows_off,
                   urows + inst.urows_off, X + inst.x_off, smem);
}

// x <- A^{-T} x with the same LU (SparseMatrix::solve_transposed).
__global__ void __launch_bounds__(256)
solve_transposed_kernel(const PlanDesc* __restrict__ plans, const int32_t* __restrict__ pool,
                        const InstDesc* __restrict__ insts, const double* __restrict__ LU,
                        double* __restrict__ X, double* __restrict__ W) {
    const InstDesc inst = insts[blockIdx.x];
    cta_solve_transposed(plans[inst.plan], pool, LU + inst.lu_off, X + inst.x_off, W + inst.w_off);
}

// max_col / max_n: largest LU column and order over the batch's plans.
cudaError_t launch_refactor(const PlanDesc* plans, const int32_t* pool, const InstDesc* insts,
                            int count, const double* A, double* LU, double diag_gmin,
                            int check_pivots, double rel_threshold, int32_t* status,
                            int32_t* fail_step, int max_col, int max_n, bool allow_flow,
                            double* lrows, double* urows, cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    const int colbuf = (max_col + 31) & ~31;
    const size_t smem = flow_smem_bytes(colbuf, max_n);
    if (allow_flow && smem <= 200 * 1024) {
        static bool configured = false;
        if (!configured) {
            cudaError_t e = cudaFuncSetAttribute(refactor_flow_kernel,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 200 * 1024);
            if (e != cudaSuccess) return e;
            configured = true;
        }
        refactor_flow_kernel<<<count, kFlowThreads, smem, stream>>>(
            plans, pool, insts, A, LU, diag_gmin, check_pivots, rel_threshold, status, fail_step,
            colbuf, lrows, urows);
    } else {
        refactor_kernel<<<count, 256, 0, stream>>>(plans, pool, insts, A, LU, diag_gmin,
                                                   check_pivots, rel_threshold, status, fail_step);
    }
    return cudaGetLastError();
}

cudaError_t launch_solve(const PlanDesc* plans, const int32_t* pool, const InstDesc* insts,
                         int count, const double* LU, double* X, double* W, bool transposed,
                         const double* lrows, const double* urows, int max_n,
                         cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    const size_t smem = flow_solve_smem_bytes(max_n);
    if (!transposed && lrows && smem <= 200 * 1024) {
        static bool configured = false;
        if (!configured) {
            cudaError_t e = cudaFuncSetAttribute(solve_flow_kernel,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 200 * 1024);
            if (e != cudaSuccess) return e;
            configured = true;
        }
        solve_flow_kernel<<<count, kFlowThreads, smem, stream>>>(plans, pool, insts, LU, lrows,
                                                                  urows, X);
        return cudaGetLastError();
    }
    if (transposed)
        solve_transposed_kernel<<<count, 256, 0, stream>>>(plans, pool, insts, LU, X, W);
    else
        solve_kernel<<<count, 256, 0, stream>>>(plans, pool, insts, LU, X, W);
    return cudaGetLastError();
}

}  // namespace nsg
