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

// Asynchronous global -> shared copies (LDGSTS).  The 16-byte form goes
// through L2 only (.cg), so, like ld.global.cg, it never sees a stale L1
// line of a column another SM finished; the 4-byte form (.ca) is used only
// for the plan's read-only index arrays.
__device__ __forceinline__ void cp_async16_cg(void* sdst, const void* gsrc) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(sdst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async4_ca(void* sdst, const void* gsrc) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(sdst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
// Wait until at most `pending` of this thread's most recent copy groups are
// still in flight (pending < kCtaRing).
__device__ __forceinline__ void cp_async_wait(int pending) {
    switch (pending) {
        case 0: asm volatile("cp.async.wait_group 0;" ::: "memory"); break;
        case 1: asm volatile("cp.async.wait_group 1;" ::: "memory"); break;
        case 2: asm volatile("cp.async.wait_group 2;" ::: "memory"); break;
        case 3: asm volatile("cp.async.wait_group 3;" ::: "memory"); break;
        case 4: asm volatile("cp.async.wait_group 4;" ::: "memory"); break;
        case 5: asm volatile("cp.async.wait_group 5;" ::: "memory"); break;
        case 6: asm volatile("cp.async.wait_group 6;" ::: "memory"); break;
        default: asm volatile("cp.async.wait_group 7;" ::: "memory"); break;
    }
}

}  // namespace

// Tail columns by whole CTAs.  The last columns of an elimination (the top
// separators) each apply hundreds to thousands of updates, and they form a
// chain: one warp per column leaves most of the GPU idle while each tail
// column works through its updates one L2 round trip at a time.  Columns
// from cta_from on are instead claimed by whole CTAs: the rows of L(:, r)
// of each update are spread over all threads, and the next kCtaRing
// updates' L(:, r) rows (up to kCtaSlot each) and destinations are staged
// into shared memory by cp.async as soon as warp 0 has seen their source
// columns complete (one batched poll of several flags), so an update costs
// two CTA barriers instead of a round trip.  Every entry still receives its
// updates in the column's stored order, one at a time, with the same
// operations: values are those of refactor_column.
constexpr int kCtaRing = 8;      // updates staged ahead
constexpr int kCtaSlot = 1024;   // rows of L(:, r) staged per update
constexpr int kCtaBuf = 8192;    // the column's shared buffer (longer: in place in lu)

struct CtaRing {
    double val[kCtaRing][kCtaSlot + 2];  // 16-byte aligned pairs, from the aligned start
    int32_t dst[kCtaRing][kCtaSlot];     // update map entries, or L(:, r)'s row indices
};

__host__ __device__ constexpr size_t cta_smem_bytes() {
    return sizeof(double) * kCtaBuf + sizeof(CtaRing);
}

struct CtaShared {
    int32_t j, nstage, timeout;
    ColumnResult res;
    AmdCand part[32];  // per-warp pivot candidates
};


struct GridState {
    int32_t next;                  // claim counter
    int32_t timeout;               // a bounded wait gave up
    int32_t growth;                // AMD-LU: a replay growth test failed
    int32_t next_cta;              // claim counter of the CTA-mode tail
    unsigned long long fail_inv;   // max of ~fail_key over failing columns (0: none)
};

// Column j of an AMD-LU plan by the whole CTA (kThreads threads); buf is
// kCtaBuf doubles of shared memory or the column's place in lu.  Same
// result as refactor_column<true> for the same column.
template <int kThreads>
__device__ ColumnResult refactor_column_cta(const PlanDesc& pd, const int32_t* __restrict__ pool,
                                            const double* __restrict__ a, double* lu,
                                            double diag_gmin, int check_pivots, int32_t j,
                                            double* buf, double* lrows, double* urows,
                                            const int32_t* done, int32_t* rmap, CtaRing& ring,
                                            CtaShared& sh) {
    const int32_t* col_ptr = pool + pd.off[PA_col_ptr];
    const int32_t* diag_pos = pool + pd.off[PA_diag_pos];
    const int32_t* lu_src = pool + pd.off[PA_lu_src];
    const int32_t* upd_dst = pool + pd.off[PA_upd_dst];
    const int32_t map16 = pd.map16;
    const int32_t* row_idx = pool + pd.off[PA_row_idx];
    const int32_t* piv_rank = pool + pd.off[PA_piv_rank];
    const int32_t* gmin_pos = pool + pd.off[PA_gmin_pos];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int32_t c0 = col_ptr[j];
    const int32_t len = col_ptr[j + 1] - c0;
    const int32_t dj = diag_pos[j] - c0;
    const int32_t gp = gmin_pos[j];
    const bool mapped = rmap == nullptr;
    for (int32_t t = tid; t < len; t += kThreads) {
        const int32_t s = lu_src[c0 + t];
        double v = (s >= 0) ? a[s] : 0.0;
        if (t == gp && diag_gmin != 0.0) v = __dadd_rn(v, diag_gmin);
        buf[t] = v;
        if (!mapped) rmap[row_idx[c0 + t]] = t;
    }
    const int4* umeta = reinterpret_cast<const int4*>(pool + pd.off[PA_umeta]) + c0;
    if (tid == 0) sh.timeout = 0;
    __syncthreads();
    // L(:, r) of update q from its 16-byte aligned start: the pair holding
    // row l0 may begin one value early (the pivot of column r); a last value
    // without its pair is read directly when applied.
    auto span = [&](const int4& m, int32_t& l0, int32_t& ns, int& off) {
        l0 = m.y + 1;
        ns = m.z < kCtaSlot ? m.z : kCtaSlot;
        off = static_cast<int>((reinterpret_cast<uintptr_t>(lu + l0) >> 3) & 1);
    };
    auto stage = [&](int32_t q) {
        const int4 m = umeta[q];
        const int slot = q % kCtaRing;
        int32_t l0, ns;
        int off;
        span(m, l0, ns, off);
        const double* g0 = lu + l0 - off;
        const int32_t pairs = (off + ns) >> 1;
        for (int32_t p = tid; p < pairs; p += kThreads)
            cp_async16_cg(&ring.val[slot][2 * p], g0 + 2 * p);
        if (mapped && map16) {
            // packed map: the words holding positions m.w .. m.w + ns - 1,
            // from the even position at or below m.w (4-byte aligned)
            const int32_t* src = reinterpret_cast<const int32_t*>(
                reinterpret_cast<const uint16_t*>(upd_dst) + (m.w & ~1));
            const int32_t words = ((m.w & 1) + ns + 1) >> 1;
            for (int32_t k = tid; k < words; k += kThreads) cp_async4_ca(&ring.dst[slot][k], src + k);
        } else {
            const int32_t* src = mapped ? upd_dst + m.w : row_idx + l0;
            for (int32_t k = tid; k < ns; k += kThreads) cp_async4_ca(&ring.dst[slot][k], src + k);
        }
        cp_async_commit();
    };
    double colmax = 0.0;  // the same in every thread: largest |U(r, j)| applied
    int32_t staged = 0;   // updates whose copies are issued
    bool timed_out = false;
    for (int32_t q = 0; q < dj; ++q) {
        if (staged < dj && staged - q <= kCtaRing / 2) {
            // warp 0 polls the flags of the next updates at once and the
            // CTA stages the prefix whose source columns are done; update
            // q itself is waited for when nothing is staged for it
            const int32_t want = ((dj < q + kCtaRing) ? dj : q + kCtaRing) - staged;
            if (warp == 0) {
                const bool ready =
                    lane < want && gflag_acquire(done + umeta[staged + lane].x) >= 1;
                const unsigned mask = __ballot_sync(0xffffffffu, ready);
                int32_t nready = __ffs(~mask) - 1;
                if (nready > want) nready = want;
                if (nready == 0 && staged == q) {
                    int ok = 1;
                    if (lane == 0) ok = gwait(done + umeta[q].x, 1) ? 1 : 0;
                    ok = __shfl_sync(0xffffffffu, ok, 0);
                    nready = ok;
                    if (!ok && lane == 0) sh.timeout = 1;
                }
                if (lane == 0) sh.nstage = nready;
            }
            __syncthreads();
            if (sh.timeout) {
                timed_out = true;
                break;
            }
            const int32_t nst = sh.nstage;
            for (int32_t i = 0; i < nst; ++i) stage(staged + i);
            staged += nst;
        }
        cp_async_wait(staged - q - 1);
        __syncthreads();
        const int4 m = umeta[q];
        const int slot = q % kCtaRing;
        int32_t l0, ns;
        int off;
        span(m, l0, ns, off);
        const double u = buf[q];
        colmax = fmax(colmax, fabs(u));
        const bool tail = ((off + ns) & 1) != 0;
        const uint16_t* dst16 = reinterpret_cast<const uint16_t*>(ring.dst[slot]) + (m.w & 1);
        const bool packed = mapped && map16;
        for (int32_t k = tid; k < ns; k += kThreads) {
            const double lv = (tail && k == ns - 1) ? __ldcg(lu + l0 + k) : ring.val[slot][off + k];
            const int32_t d = packed ? static_cast<int32_t>(dst16[k])
                                     : (mapped ? ring.dst[slot][k] : rmap[ring.dst[slot][k]]);
            buf[d] = lu_sub(buf[d], lu_mul(u, lv));
        }
        for (int32_t k = ns + tid; k < m.z; k += kThreads) {
            const int32_t d = mapped ? upd_at(upd_dst, map16, m.w + k) : rmap[row_idx[l0 + k]];
            buf[d] = lu_sub(buf[d], lu_mul(u, __ldcg(lu + l0 + k)));
        }
        __syncthreads();  // the column's new values before the next u; slot q free
    }
    cp_async_wait(0);
    __syncthreads();
    // amd_column_status with the candidate search spread over the CTA
    const bool scan = check_pivots == kCheckNumeric || check_pivots == kCheckRefactor;
    AmdCand cand{-1.0, INT32_MAX, -1};
    if (scan) {
        cand = amd_cand_warp(amd_cand_scan(buf, dj, len, piv_rank[j], tid, kThreads));
        if (lane == 0) sh.part[warp] = cand;
        __syncthreads();
    }
    if (tid == 0) {
        if (scan)
            for (int w = 1; w < kThreads / 32; ++w)
                amd_cand_merge(cand, sh.part[w].best, sh.part[w].rank, sh.part[w].pos);
        const AmdColumn v = amd_verdict(buf, dj, colmax, check_pivots, gp, cand);
        sh.res.code = v.code;
        sh.res.growth_fail = v.growth_fail;
    }
    __syncthreads();
    const ColumnResult res{sh.res.code, sh.res.growth_fail, timed_out};
    const double piv = buf[dj];
    const int32_t* rowcopy = pool + pd.off[PA_rowcopy_pos];
    for (int32_t t = tid; t < len; t += kThreads) {
        const double v = lu_store_value(true, buf[t], t, dj, piv);
        lu[c0 + t] = v;
        if (lrows) {
            if (t < dj) urows[rowcopy[c0 + t]] = v;
            else if (t > dj) lrows[rowcopy[c0 + t]] = v;
        }
    }
    __syncthreads();
    return res;
}

// kWarps warps per CTA, each with a shared column buffer of kColbuf doubles
// (columns longer than that are eliminated in place in lu).  Columns from
// cta_from on (AMD-LU plans, kColbuf >= 2048) are claimed by whole CTAs
// once all of a CTA's warps have run out of warp-mode columns; a CTA-mode
// column waits only on columns claimed earlier, so the schedule still needs
// no residency guarantee.
template <int kWarps, int kColbuf>
__global__ void __launch_bounds__(kWarps * 32)
grid_refactor_kernel(const PlanDesc* __restrict__ plans, const int32_t* __restrict__ pool,
                     const InstDesc* __restrict__ insts, int inst, const double* __restrict__ A,
                     double* LU, double diag_gmin, int check_pivots, double rel_threshold,
                     double* lrows, double* urows, int32_t* done, GridState* st,
                     int32_t* rmaps, int64_t rmap_words, int32_t cta_from) {
    extern __shared__ __align__(16) double smem[];  // 16-byte cp.async destinations
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
    const int32_t warp_end = pd.n < cta_from ? pd.n : cta_from;
    for (;;) {
        int32_t j = 0;
        if (lane == 0) j = atomicAdd(&st->next, 1);
        j = __shfl_sync(0xffffffffu, j, 0);
        if (j >= warp_end) break;
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
    if constexpr (kColbuf >= 2048) {
        if (warp_end < pd.n) {
            __shared__ CtaShared sh;
            __syncthreads();
            CtaRing& ring = *reinterpret_cast<CtaRing*>(smem + kCtaBuf);
            int32_t* crmap =
                rmaps ? rmaps + static_cast<int64_t>(blockIdx.x) * kWarps * rmap_words : nullptr;
            const double* a = A + id.a_off;
            for (;;) {
                if (threadIdx.x == 0) sh.j = warp_end + atomicAdd(&st->next_cta, 1);
                __syncthreads();
                const int32_t j = sh.j;
                if (j >= pd.n) break;
                const int32_t len = col_ptr[j + 1] - col_ptr[j];
                double* buf = (len <= kCtaBuf) ? smem : lu + col_ptr[j];
                const ColumnResult c = refactor_column_cta<kWarps * 32>(
                    pd, pool, a, lu, diag_gmin, check_pivots, j, buf, lr, ur, done, crmap, ring, sh);
                // refactor_column_cta ends with a CTA barrier after the
                // column's stores; thread 0's fence then publishes them (the
                // barrier-then-fence pattern of a grid-wide barrier)
                if (threadIdx.x == 0) {
                    __threadfence();
                    if (c.timed_out) atomicExch(&st->timeout, 1);
                    else if (c.code != kStatusOk) atomicMax(&st->fail_inv, ~fail_key(j, c.code));
                    if (c.growth_fail) atomicExch(&st->growth, 1);
                    gflag_release(done + j, 1);
                }
            }
        }
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

// Dynamic shared memory of a refactor variant: the warps' column buffers,
// or the CTA-mode column buffer and staging ring if larger.
template <int kWarps, int kColbuf>
constexpr size_t grid_refactor_smem() {
    return (kColbuf >= 2048 && cta_smem_bytes() > sizeof(double) * kWarps * kColbuf)
               ? cta_smem_bytes()
               : sizeof(double) * kWarps * kColbuf;
}

template <int kWarps, int kColbuf>
int grid_refactor_blocks() {
    static int blocks = 0;
    if (blocks == 0) {
        const size_t smem = grid_refactor_smem<kWarps, kColbuf>();
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
                                 const int32_t* cta_from_of, cudaStream_t stream) {
    colbuf = grid_colbuf(colbuf, max_col);
    int blocks = 0, threads = 0;
    size_t smem = 0;
    if (colbuf == 1024) {
        blocks = grid_refactor_blocks<8, 1024>();
        threads = 256;
        smem = grid_refactor_smem<8, 1024>();
    } else if (colbuf == 2048) {
        blocks = grid_refactor_blocks<8, 2048>();
        threads = 256;
        smem = grid_refactor_smem<8, 2048>();
    } else if (colbuf == 4096) {
        blocks = grid_refactor_blocks<4, 4096>();
        threads = 128;
        smem = grid_refactor_smem<4, 4096>();
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
            done, st, rmaps, rmap_words, colbuf >= 2048 ? cta_from_of[i] : n_of[i])
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
