// Batched complex refactor and solve for AC sweeps: every instance of a batch
// (typically one frequency point of G + jwC, or one circuit) refactored with
// the fixed pivot order of the plan -- SparseMatrix::factor_complex
// (src/solver/factor.cpp:1054-1141) -- and swept -- solve_complex
// (src/solver/solve.cpp:49-100).  Values are interleaved (re, im) per matrix
// slot / LU position / unknown.  Every complex product keeps the reference's
// grouping (re = a*c - b*d, im = a*d + b*c, one rounding each), and every
// entry receives its updates in ascending pivot order, so the factors and
// solutions are bit-identical to the reference's under the same pivots.
#include "lu_cta.cuh"

#include <cuda_runtime.h>

namespace nsg {

namespace {

constexpr int kCplxWarps = 8;
constexpr int kCplxThreads = kCplxWarps * 32;

// complex_ops::reciprocal (src/solver/element.hpp:42-54).
__device__ __forceinline__ void c_recip(double den_r, double den_i, double& out_r,
                                        double& out_i) {
    if ((den_r >= den_i && den_r > -den_i) || (den_r < den_i && den_r <= -den_i)) {
        const double r = __ddiv_rn(den_i, den_r);
        out_r = __ddiv_rn(1.0, __dadd_rn(den_r, __dmul_rn(r, den_i)));
        out_i = __dmul_rn(-r, out_r);
    } else {
        const double r = __ddiv_rn(den_r, den_i);
        out_i = __ddiv_rn(-1.0, __dadd_rn(den_i, __dmul_rn(r, den_r)));
        out_r = __dmul_rn(-r, out_i);
    }
}

// a*c - b*d and a*d + b*c with separately rounded products.
__device__ __forceinline__ double c_re(double a, double b, double c, double d) {
    return __dsub_rn(__dmul_rn(a, c), __dmul_rn(b, d));
}
__device__ __forceinline__ double c_im(double a, double b, double c, double d) {
    return __dadd_rn(__dmul_rn(a, d), __dmul_rn(b, c));
}

// One CTA per instance; warps claim columns in pivot order and eliminate each
// in place in lu (interleaved complex), waiting (bounded) for the columns
// their U entries name.  Completion flags live in shared memory.
__global__ void __launch_bounds__(kCplxThreads)
complex_refactor_kernel(const PlanDesc* __restrict__ plans, const int32_t* __restrict__ pool,
                        const InstDesc* __restrict__ insts, const double* __restrict__ A,
                        double* LU, int32_t* status) {
    extern __shared__ int32_t s_done[];
    __shared__ int32_t s_next, s_fail, s_timeout;
    const InstDesc id = insts[blockIdx.x];
    const PlanDesc& pd = plans[id.plan];
    const int32_t n = pd.n;
    const int32_t* col_ptr = pool + pd.off[PA_col_ptr];
    const int32_t* diag_pos = pool + pd.off[PA_diag_pos];
    const int32_t* lu_src = pool + pd.off[PA_lu_src];
    const int32_t* upd_dst = pool + pd.off[PA_upd_dst];
    const int32_t map16 = pd.map16;
    const int4* umeta = reinterpret_cast<const int4*>(pool + pd.off[PA_umeta]);
    const double* a = A + 2 * id.a_off;
    double* lu = LU + 2 * id.lu_off;
    const int lane = threadIdx.x & 31;
    for (int32_t j = threadIdx.x; j < n; j += blockDim.x) s_done[j] = 0;
    if (threadIdx.x == 0) {
        s_next = 0;
        s_fail = 0x7fffffff;
        s_timeout = 0;
    }
    __syncthreads();
    const int limit = c_wait_limit;
    for (;;) {
        int32_t j = 0;
        if (lane == 0) j = atomicAdd(&s_next, 1);
        j = __shfl_sync(0xffffffffu, j, 0);
        if (j >= n) break;
        const int32_t c0 = col_ptr[j];
        const int32_t len = col_ptr[j + 1] - c0;
        const int32_t dj = diag_pos[j] - c0;
        double* col = lu + 2 * static_cast<int64_t>(c0);
        for (int32_t t = lane; t < len; t += 32) {
            const int32_t src = lu_src[c0 + t];
            col[2 * t] = src >= 0 ? a[2 * src] : 0.0;
            col[2 * t + 1] = src >= 0 ? a[2 * src + 1] : 0.0;
        }
        __syncwarp();
        bool timed_out = false;
        for (int32_t q = 0; q < dj; ++q) {
            const int4 m = umeta[c0 + q];  // {r, diag_pos[r], |L(:, r)|, upd_start}
            int ready = 0;
            if (lane == 0) {
                int spins = 0;
                while ((ready = flag_acquire(s_done + m.x)) == 0) {
                    if (++spins > limit) break;
                    __nanosleep(32);
                }
            }
            ready = __shfl_sync(0xffffffffu, ready, 0);
            if (!ready) {
                timed_out = true;
                break;
            }
            const double pr = lu[2 * static_cast<int64_t>(m.y)];
            const double pi = lu[2 * static_cast<int64_t>(m.y) + 1];
            const double xr = col[2 * q], xi = col[2 * q + 1];
            const double ur = c_re(xr, xi, pr, pi);
            const double ui = c_im(xr, xi, pr, pi);
            __syncwarp();
            if (lane == 0) {
                col[2 * q] = ur;
                col[2 * q + 1] = ui;
            }
            const double* lcol = lu + 2 * (static_cast<int64_t>(m.y) + 1);
            for (int32_t t = lane; t < m.z; t += 32) {
                const int32_t dst = upd_at(upd_dst, map16, m.w + t);
                const double lr = lcol[2 * t], li = lcol[2 * t + 1];
                col[2 * dst] = __dsub_rn(col[2 * dst], c_re(ur, ui, lr, li));
                col[2 * dst + 1] = __dsub_rn(col[2 * dst + 1], c_im(ur, ui, lr, li));
            }
            __syncwarp();
        }
        if (lane == 0) {
            if (timed_out) {
                s_timeout = 1;
            } else {
                const double vr = col[2 * dj], vi = col[2 * dj + 1];
                if (__dadd_rn(fabs(vr), fabs(vi)) == 0.0) {
                    atomicMin(&s_fail, j);
                } else {
                    double rr, ri;
                    c_recip(vr, vi, rr, ri);
                    col[2 * dj] = rr;
                    col[2 * dj + 1] = ri;
                }
            }
            __threadfence_block();
            flag_release(s_done + j, 1);
        }
        __syncwarp();
    }
    __syncthreads();
    if (threadIdx.x == 0)
        status[id.index] = s_timeout ? kStatusTimeout
                                     : (s_fail != 0x7fffffff ? kStatusSingular : kStatusOk);
}

// x <- A^{-1} x for one instance per CTA, level-synchronous: rows of a level
// in parallel, each accumulating its updates in the reference's order
// (forward: columns ascending, skipping zero x_c; backward: row dot in
// ascending column order).  w: 2n doubles of scratch.
__global__ void __launch_bounds__(kCplxThreads)
complex_solve_kernel(const PlanDesc* __restrict__ plans, const int32_t* __restrict__ pool,
                     const InstDesc* __restrict__ insts, const double* __restrict__ LU,
                     double* X, double* W) {
    const InstDesc id = insts[blockIdx.x];
    const PlanDesc& pd = plans[id.plan];
    const int32_t n = pd.n;
    const int32_t* perm_row = pool + pd.off[PA_perm_row];
    const int32_t* perm_col = pool + pd.off[PA_perm_col];
    const int32_t* diag_pos = pool + pd.off[PA_diag_pos];
    const double* lu = LU + 2 * id.lu_off;
    double* x = X + 2 * id.x_off;
    double* w = W + 2 * id.w_off;
    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) {
        w[2 * i] = x[2 * perm_row[i]];
        w[2 * i + 1] = x[2 * perm_row[i] + 1];
    }
    __syncthreads();
    {
        const int32_t* lp = pool + pd.off[PA_lrow_ptr];
        const int32_t* lpos = pool + pd.off[PA_lrow_pos];
        const int32_t* lcol = pool + pd.off[PA_lrow_col];
        const int32_t* lev_ptr = pool + pd.off[PA_fwd_lev_ptr];
        const int32_t* lev = pool + pd.off[PA_fwd_lev];
        for (int32_t l = 0; l < pd.n_fwd_lev; ++l) {
            for (int32_t k = lev_ptr[l] + threadIdx.x; k < lev_ptr[l + 1]; k += blockDim.x) {
                const int32_t i = lev[k];
                double tr = w[2 * i], ti = w[2 * i + 1];
                for (int32_t e = lp[i]; e < lp[i + 1]; ++e) {
                    const int32_t c = lcol[e];
                    const double xr = w[2 * c], xi = w[2 * c + 1];
                    if (xr != 0.0 || xi != 0.0) {
                        const double lr = lu[2 * lpos[e]], li = lu[2 * lpos[e] + 1];
                        tr = __dsub_rn(tr, c_re(xr, xi, lr, li));
                        ti = __dsub_rn(ti, c_im(xr, xi, lr, li));
                    }
                }
                if (tr != 0.0 || ti != 0.0) {
                    const double pr = lu[2 * diag_pos[i]], pi = lu[2 * diag_pos[i] + 1];
                    const double nr = c_re(tr, ti, pr, pi);
                    ti = c_im(tr, ti, pr, pi);
                    tr = nr;
                }
                w[2 * i] = tr;
                w[2 * i + 1] = ti;
            }
            __syncthreads();
        }
    }
    {
        const int32_t* up = pool + pd.off[PA_urow_ptr];
        const int32_t* upos = pool + pd.off[PA_urow_pos];
        const int32_t* ucol = pool + pd.off[PA_urow_col];
        const int32_t* lev_ptr = pool + pd.off[PA_bwd_lev_ptr];
        const int32_t* lev = pool + pd.off[PA_bwd_lev];
        for (int32_t l = 0; l < pd.n_bwd_lev; ++l) {
            for (int32_t k = lev_ptr[l] + threadIdx.x; k < lev_ptr[l + 1]; k += blockDim.x) {
                const int32_t i = lev[k];
                double tr = w[2 * i], ti = w[2 * i + 1];
                for (int32_t e = up[i]; e < up[i + 1]; ++e) {
                    const int32_t c = ucol[e];
                    const double ur = lu[2 * upos[e]], ui = lu[2 * upos[e] + 1];
                    const double xr = w[2 * c], xi = w[2 * c + 1];
                    tr = __dsub_rn(tr, c_re(ur, ui, xr, xi));
                    ti = __dsub_rn(ti, __dadd_rn(__dmul_rn(ur, xi), __dmul_rn(ui, xr)));
                }
                w[2 * i] = tr;
                w[2 * i + 1] = ti;
            }
            __syncthreads();
        }
    }
    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) {
        x[2 * perm_col[i]] = w[2 * i];
        x[2 * perm_col[i] + 1] = w[2 * i + 1];
    }
}

}  // namespace

// Shared memory of the complex refactor: the completion flags.
size_t complex_refactor_smem(int max_n) { return sizeof(int32_t) * static_cast<size_t>(max_n); }

cudaError_t launch_complex_refactor(const PlanDesc* plans, const int32_t* pool,
                                    const InstDesc* insts, int count, int max_n, const double* A,
                                    double* LU, int32_t* status, cudaStream_t stream) {
    const size_t smem = complex_refactor_smem(max_n);
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(
            complex_refactor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
    }
    complex_refactor_kernel<<<count, kCplxThreads, smem, stream>>>(plans, pool, insts, A, LU,
                                                                    status);
    return cudaGetLastError();
}

cudaError_t launch_complex_solve(const PlanDesc* plans, const int32_t* pool, const InstDesc* insts,
                                 int count, const double* LU, double* X, double* W,
                                 cudaStream_t stream) {
    complex_solve_kernel<<<count, kCplxThreads, 0, stream>>>(plans, pool, insts, LU, X, W);
    return cudaGetLastError();
}

}  // namespace nsg
