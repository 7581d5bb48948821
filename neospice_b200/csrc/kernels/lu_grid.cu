// Grid-wide refactor and sweeps: one large instance at a time, every SM
// working on it.  The batched kernels give each instance one CTA, which is
// right for thousands of small circuits but leaves a single large topology
// (a power grid of 10^5 unknowns) on one SM.  Here the columns (rows) of one
// instance are claimed by warps (threads) of a persistent grid from a global
// counter in pivot (level) order, and every dependency is a completion flag
// in global memory: written with st.release.gpu after the column's values,
// read with ld.acquire.gpu before them, with the values themselves read
// L2-only (ld.global.cg) so no SM sees a stale L1 line of a column another SM
// finished.  Columns are only claimed by running warps and only wait on
// earlier claims, so the schedule cannot deadlock whatever the residency;
// every wait is still bounded (c_wait_limit polls) and reports kStatusTimeout.
//
// The per-column work is refactor_column (lu_cta.cuh), so values and their
// rounding are those of the batched kernels: bit-identical to the
// reference's SparseMatrix::factor / AmdLuSolver replay under the same
// pivots.  A column longer than the shared-memory buffer is eliminated in
// place in the LU array.
#include "lu_cta.cuh"

#include <cuda_runtime.h>

namespace nsg {

namespace {

constexpr int kGridWarps = 8;    // warps per CTA of the grid-wide sweeps
// Rounds of 32 rows of L(:, r) a warp loads before applying them: long L
// columns (the separators' hundreds of rows) then cost one L2 round trip
// per 512 rows instead of per 128.
constexpr int kGridChunk = 16;
constexpr int kGridThreads = kGridWarps * 32;

__device__ __forceinline__ int32_t gflag_acquire(const int32_t* f) {
    int32_t v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(f) : "memory");
    return v;
}

__device__ __forceinline__ void gflag_release(int32_t* f, int32_t v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(f), "r"(v) : "memory");
}

// Bounded wait until *f >= target; false on timeout.
__device__ __forceinline__ bool gwait(const int32_t* f, int32_t target) {
    if (gflag_acquire(f) >= target) return true;
    const int limit = c_wait_limit;
    for (int spins = 0; spins < limit; ++spins) {
        __nanosleep(64);
        if (gflag_acquire(f) >= target) return true;
    }
    return false;
}

}  // namespace

// Shared state of one grid-wide launch, zeroed by the host before it.
struct GridState {
    int32_t next;                  // claim counter
    int32_t timeout;               // a bounded wait gave up
    int32_t growth;                // AMD-LU: a replay growth test failed
    int32_t pad;
    unsigned long long fail_inv;   // max of ~fail_key over failing columns (0: none)
};

// kWarps warps per CTA, each with a shared column buffer of kColbuf doubles
// (columns longer than that are eliminated in place in lu).
template <int kWarps, int kColbuf>
__global__ void __launch_bounds__(kWarps * 32)
grid_refactor_kernel(const PlanDesc* __restrict__ plans, const int32_t* __restrict__ pool,
                     const InstDesc* __restrict__ insts, int inst, const double* __restrict__ A,
                     double* LU, double diag_gmin, int check_pivots, double rel_threshold,
                     double* lrows, double* urows, int32_t* done, GridState* st,
                     int32_t* rmaps, int64_t rmap_words) {
    extern __shared__ double smem[];
    const InstDesc id = insts[inst];
    const PlanDesc& pd = plans[id.plan];
    const int32_t* col_ptr = pool + pd.off[PA_col_ptr];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    double* sbuf = smem + warp * kColbuf;
    // row -> position scratch of this warp (plans without an update map)
    int32_t* rmap = rmaps ? rmaps + (static_cast<int64_t>(blockIdx.x) * kWarps + warp) * rmap_words
                          : nullptr;
    double* lu = LU + id.lu_off;
    double* lr = lrows ? lrows + id.lrows_off : nullptr;
    double* ur = urows ? urows + id.urows_off : nullptr;
    for (;;) {
        int32_t j = 0;
        if (lane == 0) j = atomicAdd(&st->next, 1);
        j = __shfl_sync(0xffffffffu, j, 0);
        if (j >= pd.n) break;
        const int32_t len = col_ptr[j + 1] - col_ptr[j];
        double* buf = (len <= kColbuf) ? sbuf : lu + col_ptr[j];
        auto probe = [&](int32_t r) { return gflag_acquire(done + r); };
        const ColumnResult c = refactor_column<true, decltype(probe), kGridChunk>(
            pd, pool, A + id.a_off, lu, diag_gmin, check_pivots, rel_threshold, j, buf, lr, ur,
            probe, rmap);
        __threadfence();
        __syncwarp();
        if (lane == 0) {
            if (c.timed_out) atomicExch(&st->timeout, 1);
            else if (c.code != kStatusOk) atomicMax(&st->fail_inv, ~fail_key(j, c.code));
            if (c.growth_fail) atomicExch(&st->growth, 1);
            gflag_release(done + j, 1);
        }
        __syncwarp();
    }
}

// Status of the instance from the launch's state (the batched kernels'
// rules: a timeout wins; an AMD-LU refactorize whose growth tests all passed
// keeps the replay).
__global__ void grid_refactor_status_kernel(const PlanDesc* __restrict__ plans,
                                            const InstDesc* __restrict__ insts, int inst,
                                            int check_pivots, const GridState* st,
                                            int32_t* status, int32_t* fail_step) {
    if (threadIdx.x != 0) return;
    const InstDesc id = insts[inst];
    const bool amd = plans[id.plan].kind == kPlanAmdLu;
    int32_t code = kStatusOk, step = -1;
    if (st->timeout) {
        code = kStatusTimeout;
    } else if (st->fail_inv != 0 && !(amd && !amd_verdict_counts(check_pivots, st->growth != 0))) {
        const unsigned long long key = ~st->fail_inv;
        code = static_cast<int32_t>(key & 0xffffffffu);
        step = static_cast<int32_t>(key >> 32);
    }
    status[id.index] = code;
    if (fail_step) fail_step[id.index] = step;
}

// One sweep of x <- A^{-1} x over the row-major L / U copies.  phase 0: the
// forward sweep (rows in fwd level order, flags set to 1; reads b through
// perm_row); phase 1: the backward sweep (bwd level order, flags set to 2;
// writes x through perm_col).  A warp claims 32 consecutive rows of the
// order; each thread waits, entry by entry, for the rows it reads.  Same
// arithmetic, in the same order per row, as cta_solve_flow.
__global__ void __launch_bounds__(kGridThreads, 4)
grid_solve_kernel(const PlanDesc* __restrict__ plans, const int32_t* __restrict__ pool,
                  const InstDesc* __restrict__ insts, int inst, const double* __restrict__ LU,
                  const double* __restrict__ lrows, const double* __restrict__ urows,
                  double* X, double* W, int32_t* done, GridState* st, int phase) {
    const InstDesc id = insts[inst];
    const PlanDesc& pd = plans[id.plan];
    const int32_t n = pd.n;
    const bool amd = pd.kind == kPlanAmdLu;
    const double* lu = LU + id.lu_off;
    double* x = X + id.x_off;
    double* w = W + id.w_off;
    const int32_t* diag_pos = pool + pd.off[PA_diag_pos];
    const int lane = threadIdx.x & 31;
    bool ok = true;
    for (;;) {
        int32_t base = 0;
        if (lane == 0) base = atomicAdd(&st->next, 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) break;
        const int32_t k = base + lane;
        if (k < n) {
            if (phase == 0) {
                const int32_t* lp = pool + pd.off[PA_lrow_ptr];
                const int32_t* lcol = pool + pd.off[PA_lrow_col];
                const double* lv = lrows + id.lrows_off;
                const int32_t i = (pool + pd.off[PA_fwd_lev])[k];
                double t = x[(pool + pd.off[PA_perm_row])[i]];
                for (int32_t e = lp[i]; e < lp[i + 1]; ++e) {
                    const int32_t c = lcol[e];
                    if (ok && !gwait(done + c, 1)) ok = false;
                    const double xc = __ldcg(w + c);
                    if (amd) t = lu_sub(t, lu_mul(lv[e], xc));
                    else if (xc != 0.0) t = lu_sub(t, lu_mul(xc, lv[e]));
                }
                if (!amd) t = (t != 0.0) ? lu_mul(t, lu[diag_pos[i]]) : t;
                __stcg(w + i, t);
                __threadfence();
                gflag_release(done + i, 1);
            } else {
                const int32_t* up = pool + pd.off[PA_urow_ptr];
                const int32_t* ucol = pool + pd.off[PA_urow_col];
                const double* uv = urows + id.urows_off;
                const int32_t i = (pool + pd.off[PA_bwd_lev])[k];
                double t = __ldcg(w + i);
                const int32_t e0 = up[i], e1 = up[i + 1];
                for (int32_t m = 0; m < e1 - e0; ++m) {
                    const int32_t e = amd ? e1 - 1 - m : e0 + m;
                    const int32_t c = ucol[e];
                    if (ok && !gwait(done + c, 2)) ok = false;
                    t = lu_sub(t, lu_mul(uv[e], __ldcg(w + c)));
                }
                if (amd) t = __ddiv_rn(t, lu[diag_pos[i]]);
                __stcg(w + i, t);
                __threadfence();
                gflag_release(done + i, 2);
                x[(pool + pd.off[PA_perm_col])[i]] = t;
            }
        }
    }
    if (!ok) atomicExch(&st->timeout, 1);
}

template <int kWarps, int kColbuf>
int grid_refactor_blocks() {
    static int blocks = 0;
    if (blocks == 0) {
        const size_t smem = sizeof(double) * kWarps * kColbuf;
        if (cudaFuncSetAttribute(grid_refactor_kernel<kWarps, kColbuf>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)) != cudaSuccess)
            return 0;
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grid_refactor_kernel<kWarps, kColbuf>,
                                                      kWarps * 32, smem);
        blocks = sms * (per_sm > 0 ? per_sm : 1);
    }
    return blocks;
}

int grid_solve_blocks() {
    static int blocks = 0;
    if (blocks == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grid_solve_kernel, kGridThreads, 0);
        blocks = sms * (per_sm > 0 ? per_sm : 1);
    }
    return blocks;
}

// Scratch of the grid-wide launches: max_n flags plus two GridStates.
size_t grid_scratch_bytes(int max_n) {
    return sizeof(GridState) * 2 + sizeof(int32_t) * static_cast<size_t>(max_n);
}

// Refactor every instance of the batch in turn with the whole GPU.  The
// per-warp column buffer: colbuf doubles (1024, 2048 or 4096; 0 = the
// smallest that holds the longest column, max_col).  1024: 8 warps and
// 64 KB per CTA, three CTAs per SM; 2048: 8 warps, 128 KB, one per SM;
// 4096: 4 warps, 128 KB.  Fewer warps in flight, but the long separator
// columns at the top of the elimination stay in shared memory instead of
// being updated in place in global memory.
static int grid_colbuf(int colbuf, int max_col) {
    return colbuf != 0 ? colbuf : (max_col <= 1024 ? 1024 : (max_col <= 2048 ? 2048 : 4096));
}

// Words of the per-warp row -> position maps a launch with these settings
// needs for plans without an update map (every warp of the grid, n words
// each).
int64_t grid_rmap_words(int colbuf, int max_col, int max_n) {
    colbuf = grid_colbuf(colbuf, max_col);
    int warps = 0;
    if (colbuf == 1024) warps = grid_refactor_blocks<8, 1024>() * 8;
    else if (colbuf == 2048) warps = grid_refactor_blocks<8, 2048>() * 8;
    else warps = grid_refactor_blocks<4, 4096>() * 4;
    return static_cast<int64_t>(warps) * max_n;
}

cudaError_t launch_grid_refactor(const PlanDesc* plans, const int32_t* pool,
                                 const InstDesc* insts, int count, const int32_t* n_of,
                                 const double* A, double* LU, double diag_gmin, int check_pivots,
                                 double rel_threshold, int32_t* status, int32_t* fail_step,
                                 double* lrows, double* urows, void* scratch, int colbuf,
                                 int max_col, int32_t* rmaps, int64_t rmap_words,
                                 cudaStream_t stream) {
    colbuf = grid_colbuf(colbuf, max_col);
    int blocks = 0, threads = 0;
    size_t smem = 0;
    if (colbuf == 1024) {
        blocks = grid_refactor_blocks<8, 1024>();
        threads = 256;
        smem = sizeof(double) * 8 * 1024;
    } else if (colbuf == 2048) {
        blocks = grid_refactor_blocks<8, 2048>();
        threads = 256;
        smem = sizeof(double) * 8 * 2048;
    } else if (colbuf == 4096) {
        blocks = grid_refactor_blocks<4, 4096>();
        threads = 128;
        smem = sizeof(double) * 4 * 4096;
    } else {
        return cudaErrorInvalidValue;
    }
    if (blocks == 0) return cudaErrorInvalidConfiguration;
    GridState* st = static_cast<GridState*>(scratch);
    int32_t* done = reinterpret_cast<int32_t*>(st + 2);
    for (int i = 0; i < count; ++i) {
        cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(GridState) * 2 +
                                                        sizeof(int32_t) * static_cast<size_t>(n_of[i]),
                                        stream);
        if (e != cudaSuccess) return e;
#define NSG_GRID_REFACTOR(W, C)                                                                \
        grid_refactor_kernel<W, C><<<blocks, threads, smem, stream>>>(                         \
            plans, pool, insts, i, A, LU, diag_gmin, check_pivots, rel_threshold, lrows, urows, \
            done, st, rmaps, rmap_words)
        if (colbuf == 1024) NSG_GRID_REFACTOR(8, 1024);
        else if (colbuf == 2048) NSG_GRID_REFACTOR(8, 2048);
        else NSG_GRID_REFACTOR(4, 4096);
#undef NSG_GRID_REFACTOR
        grid_refactor_status_kernel<<<1, 32, 0, stream>>>(plans, insts, i, check_pivots, st,
                                                          status, fail_step);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// x <- A^{-1} x for every instance in turn with the whole GPU (needs the
// row-major copies written by a dataflow or grid-wide refactor).  A bounded
// wait that gave up leaves that instance's result undefined, as in the
// batched sweeps.
cudaError_t launch_grid_solve(const PlanDesc* plans, const int32_t* pool, const InstDesc* insts,
                              int count, const int32_t* n_of, const double* LU,
                              const double* lrows, const double* urows, double* X, double* W,
                              void* scratch, cudaStream_t stream) {
    const int blocks = grid_solve_blocks();
    GridState* st = static_cast<GridState*>(scratch);
    int32_t* done = reinterpret_cast<int32_t*>(st + 2);
    for (int i = 0; i < count; ++i) {
        cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(GridState) * 2 +
                                                        sizeof(int32_t) * static_cast<size_t>(n_of[i]),
                                        stream);
        if (e != cudaSuccess) return e;
        grid_solve_kernel<<<blocks, kGridThreads, 0, stream>>>(plans, pool, insts, i, LU, lrows,
                                                               urows, X, W, done, st, 0);
        grid_solve_kernel<<<blocks, kGridThreads, 0, stream>>>(plans, pool, insts, i, LU, lrows,
                                                               urows, X, W, done, st + 1, 1);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace nsg
