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
#include "lu_device.cuh"

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

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

}  // namespace

// Load A into the LU pattern, add diag_gmin to every pivot, then eliminate
// column by column.  check_pivots != 0 applies the re-validation test of
// SparseMatrix::order_and_factor (factor.cpp:929-947): the pivot must exceed
// rel_threshold times the largest entry below it, else the instance is
// flagged kStatusReorder at that step.  Otherwise only an exact zero pivot is
// flagged (kStatusSingular), as in SparseMatrix::factor.
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
    const int32_t* lev_ptr = p[PA_col_lev_ptr];
    const int32_t* lev = p[PA_col_lev];
    const double* a = A + inst.a_off;
    double* lu = LU + inst.lu_off;

    __shared__ int32_t s_fail_step;
    __shared__ int32_t s_fail_code;
    if (threadIdx.x == 0) {
        s_fail_step = INT32_MAX;
        s_fail_code = kStatusOk;
    }

    for (int32_t q = threadIdx.x; q < pd.nnz_lu; q += blockDim.x) {
        const int32_t s = lu_src[q];
        lu[q] = (s >= 0) ? a[s] : 0.0;
    }
    __syncthreads();
    if (diag_gmin != 0.0)
        for (int32_t j = threadIdx.x; j < pd.n; j += blockDim.x)
            lu[diag_pos[j]] = __dadd_rn(lu[diag_pos[j]], diag_gmin);
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    for (int32_t l = 0; l < pd.n_col_lev; ++l) {
        for (int32_t k = lev_ptr[l] + warp; k < lev_ptr[l + 1]; k += nwarps) {
            const int32_t j = lev[k];
            const int32_t dj = diag_pos[j];
            for (int32_t q = col_ptr[j]; q < dj; ++q) {
                const int32_t r = row_idx[q];
                const double u = mul(lu[q], lu[diag_pos[r]]);
                __syncwarp();
                if (lane == 0) lu[q] = u;
                const int32_t l0 = diag_pos[r] + 1;
                const int32_t cnt = col_ptr[r + 1] - l0;
                const int32_t* dst = upd_dst + upd_start[q];
                for (int32_t t = lane; t < cnt; t += 32) {
                    const int32_t d = dst[t];
                    lu[d] = sub(lu[d], mul(u, lu[l0 + t]));
                }
                __syncwarp();
            }
            const double piv = lu[dj];
            bool fail;
            if (check_pivots) {
                double largest = 0.0;
                for (int32_t q = dj + 1 + lane; q < col_ptr[j + 1]; q += 32)
                    largest = fmax(largest, fabs(lu[q]));
                largest = warp_max(largest);
                fail = !(largest * rel_threshold < fabs(piv));
            } else {
                fail = (piv == 0.0);
            }
            __syncwarp();
            if (lane == 0) {
                if (fail) {
                    atomicMin(&s_fail_step, j);
                    s_fail_code = check_pivots ? kStatusReorder : kStatusSingular;
                }
                lu[dj] = 1.0 / piv;
            }
            __syncwarp();
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        status[blockIdx.x] = s_fail_code;
        if (fail_step) fail_step[blockIdx.x] = (s_fail_code == kStatusOk) ? -1 : s_fail_step;
    }
}

// x <- A^{-1} x with the factored LU (SparseMatrix::solve).
__global__ void __launch_bounds__(256)
solve_kernel(const PlanDesc* __restrict__ plans, const int32_t* __restrict__ pool,
             const InstDesc* __restrict__ insts, const double* __restrict__ LU,
             double* __restrict__ X, double* __restrict__ W) {
    const InstDesc inst = insts[blockIdx.x];
    const PlanDesc& pd = plans[inst.plan];
    const PlanView p(pd, pool);
    const int32_t n = pd.n;
    const double* lu = LU + inst.lu_off;
    double* x = X + inst.x_off;
    double* w = W + inst.w_off;
    const int32_t* perm_row = p[PA_perm_row];
    const int32_t* perm_col = p[PA_perm_col];
    const int32_t* diag_pos = p[PA_diag_pos];

    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) w[i] = x[perm_row[i]];
    __syncthreads();

    {   // forward: L with the reciprocal pivot, row-oriented gather
        const int32_t* lp = p[PA_lrow_ptr];
        const int32_t* lpos = p[PA_lrow_pos];
        const int32_t* lcol = p[PA_lrow_col];
        const int32_t* lev_ptr = p[PA_fwd_lev_ptr];
        const int32_t* lev = p[PA_fwd_lev];
        for (int32_t l = 0; l < pd.n_fwd_lev; ++l) {
            for (int32_t k = lev_ptr[l] + threadIdx.x; k < lev_ptr[l + 1]; k += blockDim.x) {
                const int32_t i = lev[k];
                double t = w[i];
                for (int32_t e = lp[i]; e < lp[i + 1]; ++e) {
                    const double xc = w[lcol[e]];
                    if (xc != 0.0) t = sub(t, mul(xc, lu[lpos[e]]));
                }
                w[i] = (t != 0.0) ? mul(t, lu[diag_pos[i]]) : t;
            }
            __syncthreads();
        }
    }
    {   // backward: unit-diagonal U, row dot products
        const int32_t* up = p[PA_urow_ptr];
        const int32_t* upos = p[PA_urow_pos];
        const int32_t* ucol = p[PA_urow_col];
        const int32_t* lev_ptr = p[PA_bwd_lev_ptr];
        const int32_t* lev = p[PA_bwd_lev];
        for (int32_t l = 0; l < pd.n_bwd_lev; ++l) {
            for (int32_t k = lev_ptr[l] + threadIdx.x; k < lev_ptr[l + 1]; k += blockDim.x) {
                const int32_t i = lev[k];
                double t = w[i];
                for (int32_t e = up[i]; e < up[i + 1]; ++e)
                    t = sub(t, mul(lu[upos[e]], w[ucol[e]]));
                w[i] = t;
            }
            __syncthreads();
        }
    }
    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) x[perm_col[i]] = w[i];
}

// x <- A^{-T} x with the same LU (SparseMatrix::solve_transposed).
__global__ void __launch_bounds__(256)
solve_transposed_kernel(const PlanDesc* __restrict__ plans, const int32_t* __restrict__ pool,
                        const InstDesc* __restrict__ insts, const double* __restrict__ LU,
                        double* __restrict__ X, double* __restrict__ W) {
    const InstDesc inst = insts[blockIdx.x];
    const PlanDesc& pd = plans[inst.plan];
    const PlanView p(pd, pool);
    const int32_t n = pd.n;
    const double* lu = LU + inst.lu_off;
    double* x = X + inst.x_off;
    double* w = W + inst.w_off;
    const int32_t* perm_row = p[PA_perm_row];
    const int32_t* perm_col = p[PA_perm_col];
    const int32_t* col_ptr = p[PA_col_ptr];
    const int32_t* row_idx = p[PA_row_idx];
    const int32_t* diag_pos = p[PA_diag_pos];

    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) w[i] = x[perm_col[i]];
    __syncthreads();

    {   // forward over U^T: column c gathers its U entries, rows ascending
        const int32_t* lev_ptr = p[PA_col_lev_ptr];
        const int32_t* lev = p[PA_col_lev];
        for (int32_t l = 0; l < pd.n_col_lev; ++l) {
            for (int32_t k = lev_ptr[l] + threadIdx.x; k < lev_ptr[l + 1]; k += blockDim.x) {
                const int32_t c = lev[k];
                double t = w[c];
                for (int32_t q = col_ptr[c]; q < diag_pos[c]; ++q) {
                    const double xr = w[row_idx[q]];
                    if (xr != 0.0) t = sub(t, mul(xr, lu[q]));
                }
                w[c] = t;
            }
            __syncthreads();
        }
    }
    {   // backward over L^T with the reciprocal pivot
        const int32_t* lev_ptr = p[PA_tbw_lev_ptr];
        const int32_t* lev = p[PA_tbw_lev];
        for (int32_t l = 0; l < pd.n_tbw_lev; ++l) {
            for (int32_t k = lev_ptr[l] + threadIdx.x; k < lev_ptr[l + 1]; k += blockDim.x) {
                const int32_t i = lev[k];
                double t = w[i];
                for (int32_t q = diag_pos[i] + 1; q < col_ptr[i + 1]; ++q)
                    t = sub(t, mul(lu[q], w[row_idx[q]]));
                w[i] = mul(t, lu[diag_pos[i]]);
            }
            __syncthreads();
        }
    }
    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) x[perm_row[i]] = w[i];
}

cudaError_t launch_refactor(const PlanDesc* plans, const int32_t* pool, const InstDesc* insts,
                            int count, const double* A, double* LU, double diag_gmin,
                            int check_pivots, double rel_threshold, int32_t* status,
                            int32_t* fail_step, cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    refactor_kernel<<<count, 256, 0, stream>>>(plans, pool, insts, A, LU, diag_gmin,
                                               check_pivots, rel_threshold, status, fail_step);
    return cudaGetLastError();
}

cudaError_t launch_solve(const PlanDesc* plans, const int32_t* pool, const InstDesc* insts,
                         int count, const double* LU, double* X, double* W, bool transposed,
                         cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    if (transposed)
        solve_transposed_kernel<<<count, 256, 0, stream>>>(plans, pool, insts, LU, X, W);
    else
        solve_kernel<<<count, 256, 0, stream>>>(plans, pool, insts, LU, X, W);
    return cudaGetLastError();
}

}  // namespace nsg
