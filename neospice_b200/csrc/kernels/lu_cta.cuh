// CTA-level building blocks: one thread block refactors / solves one
// instance.  Used by the standalone batched kernels (lu_kernels.cu) and by the
// fused Newton kernel (newton_dc.cu).
//
// Rounding order.  Every value is produced by the same sequence of IEEE
// double operations as the reference's SparseMatrix::factor / solve /
// solve_transposed (src/solver/factor.cpp:980-1052, solve.cpp:6-47,
// :102-141): updates into one entry are applied in ascending pivot order, one
// at a time, with separately rounded multiply and subtract (__dmul_rn,
// __dsub_rn: no FMA contraction).  Results are therefore bit-identical to the
// reference under the same pivot sequence.
#pragma once
#include "lu_device.cuh"

#include <cuda_runtime.h>

namespace nsg {

constexpr int kFlowWarps = 16;
constexpr int kFlowThreads = kFlowWarps * 32;

// Polls a bounded dependency wait makes before it gives up and its instance
// reports kStatusTimeout (a wait that finds its flag set at the first look
// makes no poll; a limit of 0 gives up at the first wait that has to poll).
// Every translation unit that includes this header keeps its own copy in
// constant memory and registers a setter; nsg_set_wait_limit writes all of
// them on the current device.
constexpr int kDefaultWaitLimit = 1 << 22;
static __constant__ int c_wait_limit = kDefaultWaitLimit;

// Host: keep `set` in the list nsg_set_wait_limit walks (defined in capi.cpp).
bool register_wait_limit_setter(cudaError_t (*set)(int polls));

namespace {
cudaError_t set_wait_limit_here(int polls) {
    return cudaMemcpyToSymbol(c_wait_limit, &polls, sizeof(int));
}
const bool wait_limit_setter_registered = register_wait_limit_setter(&set_wait_limit_here);
}  // namespace
// Rounds of 32 L(:, r) rows the dataflow refactor loads before applying them.
constexpr int kColChunk = 4;

__device__ __forceinline__ double lu_mul(double x, double y) { return __dmul_rn(x, y); }
__device__ __forceinline__ double lu_sub(double x, double y) { return __dsub_rn(x, y); }

// Completion flags in shared memory: the producer publishes with a release
// store after writing its values, the consumer reads with an acquire load
// before reading them (PTX ld.acquire / st.release at CTA scope).
__device__ __forceinline__ int32_t flag_acquire(const volatile int32_t* f) {
    int32_t v;
    const unsigned addr = static_cast<unsigned>(__cvta_generic_to_shared(const_cast<int32_t*>(f)));
    asm volatile("ld.acquire.cta.shared.b32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
    return v;
}

__device__ __forceinline__ void flag_release(volatile int32_t* f, int32_t v) {
    const unsigned addr = static_cast<unsigned>(__cvta_generic_to_shared(const_cast<int32_t*>(f)));
    asm volatile("st.release.cta.shared.b32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Verdict on column k of an AMD-LU replay, computed by one warp from the
// column's values after all its U updates (col: relative to the column
// start; dj: the pivot's position; colmax: the largest |U(r, k)| applied).
//   growth_fail (kCheckRefactor only): refactor_replay_'s growth test
//     (amd_lu_solver.cpp:250-259), u_kk == 0 or |u_kk| < 1e-3 *
//     max(colmax, |u_kk|).  On any such column the reference abandons the
//     replay and runs a full factor_ on the same values.
//   code (kCheckNumeric and kCheckRefactor): whether factor_ on these
//     values (amd_lu_solver.cpp:134-157) would pick the plan's pivot row --
//     the first candidate of largest |x| in reach order, unless the row of
//     the column's own diagonal is a candidate within 1e-3 of that maximum;
//     no candidate above zero -> kStatusSingular, another row ->
//     kStatusReorder.  When every column agrees, factor_ reproduces the
//     replay's values bit for bit, so a failed growth test costs nothing.
//   kCheckNone: code is kStatusSingular for u_kk == 0.
// Ends with __syncwarp(): the caller may overwrite the column afterwards.
struct AmdColumn {
    int32_t code;
    bool growth_fail;
};

// The pivot candidate search of amd_column_status, split so a whole CTA can
// run it: each thread scans positions dj + start, dj + start + stride, ...
// and the partial results merge in any order (largest |x|, then lowest
// rank: a total order, since ranks are distinct).
struct AmdCand {
    double best;
    int32_t rank, pos;
};

__device__ __forceinline__ void amd_cand_merge(AmdCand& a, double ob, int32_t orank,
                                               int32_t opos) {
    if (ob > a.best || (ob == a.best && orank < a.rank)) {
        a.best = ob;
        a.rank = orank;
        a.pos = opos;
    }
}

__device__ inline AmdCand amd_cand_scan(const double* col, int32_t dj, int32_t len,
                                        int32_t piv_rank, int start, int stride) {
    AmdCand c{-1.0, INT32_MAX, -1};
    for (int32_t t = dj + start; t < len; t += stride) {
        int32_t rank;
        if (t == dj) {
            if (piv_rank < 0) continue;  // the pivot was not in the reach
            rank = piv_rank;
        } else {
            const int32_t m = t - dj - 1;
            rank = (piv_rank >= 0 && m >= piv_rank) ? m + 1 : m;
        }
        amd_cand_merge(c, fabs(col[t]), rank, t);
    }
    return c;
}

__device__ __forceinline__ AmdCand amd_cand_warp(AmdCand c) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, c.best, o);
        const int32_t orank = __shfl_xor_sync(0xffffffffu, c.rank, o);
        const int32_t opos = __shfl_xor_sync(0xffffffffu, c.pos, o);
        amd_cand_merge(c, ob, orank, opos);
    }
    return c;
}

// The verdict from the column's pivot, colmax and (for kCheckNumeric /
// kCheckRefactor) the merged candidate.
__device__ inline AmdColumn amd_verdict(const double* col, int32_t dj, double colmax, int check,
                                        int32_t gpos, const AmdCand& c) {
    const double piv = col[dj];
    AmdColumn r{(piv == 0.0) ? kStatusSingular : kStatusOk, false};
    if (check == kCheckRefactor) {
        const double a = fabs(piv);
        const double cm = a > colmax ? a : colmax;
        r.growth_fail = (piv == 0.0 || (cm > 0.0 && a < 1e-3 * cm));
    }
    if (check == kCheckNumeric || check == kCheckRefactor) {
        if (c.pos < 0 || c.best <= 0.0) {
            r.code = kStatusSingular;
        } else {
            int32_t chosen = c.pos;
            if (gpos >= dj && fabs(col[gpos]) >= c.best * 1e-3) chosen = gpos;
            r.code = (chosen != dj) ? kStatusReorder : (piv == 0.0 ? kStatusSingular : kStatusOk);
        }
    }
    return r;
}

__device__ inline AmdColumn amd_column_status(const double* col, int32_t dj, int32_t len,
                                              double colmax, int check, int32_t piv_rank,
                                              int32_t gpos, int lane) {
    AmdCand c{-1.0, INT32_MAX, -1};
    if (check == kCheckNumeric || check == kCheckRefactor)
        c = amd_cand_warp(amd_cand_scan(col, dj, len, piv_rank, lane, 32));
    const AmdColumn r = amd_verdict(col, dj, colmax, check, gpos, c);
    __syncwarp();
    return r;
}

// Outcome of an AMD-LU refactor from the first column verdict that failed
// (packed by fail_key, ~0 if none) and whether any growth test failed.  A
// refactorize() whose growth tests all pass keeps the replay; otherwise, as
// for a numeric(), the first failing verdict decides.
__device__ __forceinline__ bool amd_verdict_counts(int check, bool any_growth_fail) {
    return check != kCheckRefactor || any_growth_fail;
}

// Value stored at relative position t of a finished column (pivot at dj):
// Markowitz keeps L as eliminated and stores 1 / pivot; AMD-LU divides L by
// the pivot and keeps the pivot.
__device__ __forceinline__ double lu_store_value(bool amd, double v, int32_t t, int32_t dj,
                                                 double piv) {
    if (amd) return t > dj ? __ddiv_rn(v, piv) : v;
    return t == dj ? 1.0 / piv : v;
}

// First failing column and its status, packed for one atomicMin.
__device__ __forceinline__ unsigned long long fail_key(int32_t step, int32_t code) {
    return (static_cast<unsigned long long>(static_cast<uint32_t>(step)) << 32) |
           static_cast<uint32_t>(code);
}

// Shared memory of the dataflow refactor: kFlowWarps column buffers of
// colbuf doubles, then n int32 completion flags.
__host__ __device__ inline size_t flow_smem_bytes(int colbuf, int n) {
    return sizeof(double) * kFlowWarps * colbuf + sizeof(int32_t) * n;
}

struct RefactorResult {
    int32_t code;  // kStatus*
    int32_t step;  // failing pivot step or -1
};

// Outcome of one column of the dataflow refactor.
struct ColumnResult {
    int32_t code;      // kStatusOk / kStatusSingular / kStatusReorder verdict
    bool growth_fail;  // AMD-LU kCheckRefactor: the replay's growth test failed
    bool timed_out;    // a bounded dependency wait gave up
};

// Loads of another column's factor values: through L1 when one SM owns the
// whole instance, L2-only (ld.global.cg) when columns are finished by other
// SMs and an L1 line could hold values from before their completion.
template <bool kCrossSm>
__device__ __forceinline__ double lu_peer(const double* p) {
    if constexpr (kCrossSm) return __ldcg(p);
    return *p;
}

// Column j of the left-looking dataflow refactor, by one warp.  buf holds the
// column while it is eliminated (shared memory, or the column's own place in
// lu); probe(r) reads column r's completion flag (acquire).  Loads A
// (through lu_src, diag_gmin added), applies every U entry in stored order
// after column r is done, judges the pivot (check_pivots, kCheck*), and
// writes the column (and its row-major copies) to lu.  Ends with
// __syncwarp(); the caller publishes completion.  The position in column j
// of each row of L(:, r) comes from the plan's update map, or, when rmap is
// given (always for plans without a map, pd.has_map == 0), from rmap: this
// warp's row -> position scratch (pd.n words), written for column j's rows
// first.  The row map reads L(:, r)'s row indices, which every consumer
// column of r shares, instead of a map entry per update.
template <bool kCrossSm, class Probe, int kChunk = kColChunk>
__device__ __forceinline__ ColumnResult refactor_column(
    const PlanDesc& pd, const int32_t* __restrict__ pool, const double* __restrict__ a,
    double* lu, double diag_gmin, int check_pivots, double rel_threshold, int32_t j, double* buf,
    double* __restrict__ lrows, double* __restrict__ urows, Probe probe,
    int32_t* rmap = nullptr) {
    const int32_t* col_ptr = pool + pd.off[PA_col_ptr];
    const int32_t* diag_pos = pool + pd.off[PA_diag_pos];
    const int32_t* lu_src = pool + pd.off[PA_lu_src];
    const int32_t* upd_dst = pool + pd.off[PA_upd_dst];
    const int32_t map16 = pd.map16;
    const bool amd = pd.kind == kPlanAmdLu;
    const int32_t* piv_rank = pool + pd.off[PA_piv_rank];
    const int32_t* gmin_pos = pool + pd.off[PA_gmin_pos];
    const int lane = threadIdx.x & 31;

    const int32_t c0 = col_ptr[j];
    const int32_t len = col_ptr[j + 1] - c0;
    const int32_t dj = diag_pos[j] - c0;
    const int32_t gp = amd ? gmin_pos[j] : dj;
    const int32_t* row_idx = pool + pd.off[PA_row_idx];
    const bool mapped = rmap == nullptr;
    for (int32_t t = lane; t < len; t += 32) {
        const int32_t s = lu_src[c0 + t];
        double v = (s >= 0) ? a[s] : 0.0;
        if (t == gp && diag_gmin != 0.0) v = __dadd_rn(v, diag_gmin);
        buf[t] = v;
        if (!mapped) rmap[row_idx[c0 + t]] = t;
    }
    __syncwarp();
    // Position in column j of entry t of L(:, r) (its k-th update).
    auto dest = [&](int32_t us, int32_t l0, int32_t t) -> int32_t {
        return mapped ? upd_at(upd_dst, map16, us + t) : rmap[row_idx[l0 + t]];
    };
    double colmax = 0.0;  // AMD-LU: largest |U(r, j)| applied
    // U-entry metadata {r, diag_pos[r], |L(:,r)|, upd_start} is held 32
    // entries at a time in registers (lane k holds entry base+k) and
    // broadcast by shuffle.  One-step lookahead: while the update of entry q
    // runs, the pivot reciprocal, the first 32 entries of L(:, r) and their
    // destinations for entry q+1 are loaded (when column r is done), so a
    // step waits on at most one global round trip.
    const int4* umeta = reinterpret_cast<const int4*>(pool + pd.off[PA_umeta]) + c0;
    bool timed_out = false;
    int4 chunk = make_int4(0, 0, 0, 0), next_chunk = make_int4(0, 0, 0, 0);
    if (lane < dj) chunk = umeta[lane];
    if (32 + lane < dj) next_chunk = umeta[32 + lane];
    double rd_c = 0.0, lv_c = 0.0;
    int32_t l0_c = 0, cnt_c = 0, us_c = 0, ld_c = 0;
    bool have_c = false;
    // Load the operands of entry q (metadata m) if column m.x is done, or
    // after waiting for it.
    auto fetch = [&](const int4 m, bool wait, double& rd, double& lv, int32_t& l0, int32_t& cnt,
                     int32_t& us, int32_t& ld) -> bool {
        int ready = 0;
        if (lane == 0) {
            const int limit = c_wait_limit;
            int spins = 0;
            while ((ready = probe(m.x)) == 0 && wait) {
                if (++spins > limit) {
                    timed_out = true;
                    break;
                }
                __nanosleep(64);
            }
        }
        ready = __shfl_sync(0xffffffffu, ready, 0);
        timed_out = __shfl_sync(0xffffffffu, timed_out, 0);
        __syncwarp();
        if (!ready) return false;
        rd = lu_peer<kCrossSm>(lu + m.y);
        l0 = m.y + 1;
        cnt = m.z;
        us = m.w;
        lv = (lane < cnt) ? lu_peer<kCrossSm>(lu + l0 + lane) : 0.0;
        ld = (lane < cnt) ? dest(us, l0, lane) : 0;
        return true;
    };
    auto meta = [&](int32_t q) -> int4 {
        const int k = q & 31;
        const int4 src = ((q >> 5) == 0) ? chunk : next_chunk;
        int4 m;
        m.x = __shfl_sync(0xffffffffu, src.x, k);
        m.y = __shfl_sync(0xffffffffu, src.y, k);
        m.z = __shfl_sync(0xffffffffu, src.z, k);
        m.w = __shfl_sync(0xffffffffu, src.w, k);
        return m;
    };
    int32_t base = 0;  // entry index held in chunk's lane 0
    for (int32_t q = 0; q < dj; ++q) {
        if (q - base == 32) {  // advance the register window by 32 entries
            base += 32;
            chunk = next_chunk;
            next_chunk = (base + 32 + lane < dj) ? umeta[base + 32 + lane] : make_int4(0, 0, 0, 0);
        }
        if (!have_c) {
            fetch(meta(q - base), true, rd_c, lv_c, l0_c, cnt_c, us_c, ld_c);
            if (timed_out) break;
        }
        double rd_n = 0.0, lv_n = 0.0;
        int32_t l0_n = 0, cnt_n = 0, us_n = 0, ld_n = 0;
        const bool have_n = (q + 1 < dj) &&
                            fetch(meta(q + 1 - base), false, rd_n, lv_n, l0_n, cnt_n, us_n, ld_n);
        const double u = amd ? buf[q] : lu_mul(buf[q], rd_c);
        colmax = fmax(colmax, fabs(u));
        __syncwarp();
        if (lane == 0) buf[q] = u;
        if (lane < cnt_c) buf[ld_c] = lu_sub(buf[ld_c], lu_mul(u, lv_c));
        // L(:, r) beyond its first 32 rows: destinations and values are
        // loaded kChunk rounds at a time before they are applied (the
        // destinations of one entry are distinct, so the order among them
        // does not matter).
        for (int32_t t0 = 32; t0 < cnt_c; t0 += 32 * kChunk) {
            int32_t dd[kChunk];
            double ll[kChunk];
#pragma unroll
            for (int k = 0; k < kChunk; ++k) {
                const int32_t t = t0 + 32 * k + lane;
                dd[k] = (t < cnt_c) ? dest(us_c, l0_c, t) : 0;
                ll[k] = (t < cnt_c) ? lu_peer<kCrossSm>(lu + l0_c + t) : 0.0;
            }
#pragma unroll
            for (int k = 0; k < kChunk; ++k)
                if (t0 + 32 * k + lane < cnt_c) buf[dd[k]] = lu_sub(buf[dd[k]], lu_mul(u, ll[k]));
        }
        __syncwarp();
        have_c = have_n;
        rd_c = rd_n;
        lv_c = lv_n;
        l0_c = l0_n;
        cnt_c = cnt_n;
        us_c = us_n;
        ld_c = ld_n;
    }
    const double piv = buf[dj];
    ColumnResult res{kStatusOk, false, timed_out};
    if (amd) {
        const AmdColumn v = amd_column_status(buf, dj, len, colmax, check_pivots, piv_rank[j],
                                              gmin_pos[j], lane);
        res.code = v.code;
        res.growth_fail = v.growth_fail;
    } else if (check_pivots == kCheckNumeric) {
        double largest = 0.0;
        for (int32_t t = dj + 1 + lane; t < len; t += 32) largest = fmax(largest, fabs(buf[t]));
        largest = warp_max(largest);
        res.code = !(largest * rel_threshold < fabs(piv)) ? kStatusReorder : kStatusOk;
    } else {
        res.code = (piv == 0.0) ? kStatusSingular : kStatusOk;
    }
    const int32_t* rowcopy = pool + pd.off[PA_rowcopy_pos];
    for (int32_t t = lane; t < len; t += 32) {
        const double v = lu_store_value(amd, buf[t], t, dj, piv);
        lu[c0 + t] = v;
        if (lrows) {
            if (t < dj) urows[rowcopy[c0 + t]] = v;
            else if (t > dj) lrows[rowcopy[c0 + t]] = v;
        }
    }
    __syncwarp();
    return res;
}

// Dataflow refactor of one instance by the whole CTA (blockDim.x ==
// kFlowThreads).  Warps claim columns in pivot order from a shared counter;
// before using column r a warp waits for done[r], so independent columns
// overlap and the dense trailing block pipelines as a wavefront.  Column j
// stays in a per-warp shared buffer from its load (A gathered through lu_src,
// diag_gmin added) to its write-back.  check_pivots is a kCheck* mode: for
// Markowitz plans kCheckNumeric applies the re-validation test of
// SparseMatrix::order_and_factor (factor.cpp:929-947), otherwise only an
// exact zero pivot fails, as in SparseMatrix::factor; AMD-LU plans follow
// amd_column_status.  Every
// wait is bounded: past c_wait_limit polls the instance reports kStatusTimeout
// and the warp moves on, so the CTA always finishes.  Begins and ends with
// __syncthreads().
// When lrows/urows are given, every L and U entry is also written to its
// position in the row-major copies the dataflow sweeps read.
static __device__ __noinline__ RefactorResult cta_refactor_flow(const PlanDesc& pd, const int32_t* __restrict__ pool,
                                                   const double* __restrict__ a, double* __restrict__ lu,
                                                   double diag_gmin, int check_pivots,
                                                   double rel_threshold, double* smem, int colbuf,
                                                   double* __restrict__ lrows = nullptr,
                                                   double* __restrict__ urows = nullptr,
                                                   int32_t* rmaps = nullptr,
                                                   int64_t rmap_stride = 0) {
    const int32_t n = pd.n;
    const bool amd = pd.kind == kPlanAmdLu;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    double* buf = smem + warp * colbuf;
    volatile int32_t* done = reinterpret_cast<volatile int32_t*>(smem + kFlowWarps * colbuf);
    int32_t* rmap = rmaps ? rmaps + warp * rmap_stride : nullptr;

    __shared__ int32_t s_next, s_timeout, s_growth;
    __shared__ unsigned long long s_fail;
    __syncthreads();
    for (int32_t j = threadIdx.x; j < n; j += blockDim.x) done[j] = 0;
    if (threadIdx.x == 0) {
        s_next = 0;
        s_timeout = 0;
        s_growth = 0;
        s_fail = ~0ull;
    }
    __syncthreads();

    for (;;) {
        int32_t j = 0;
        if (lane == 0) j = atomicAdd(&s_next, 1);
        j = __shfl_sync(0xffffffffu, j, 0);
        if (j >= n) break;
        const ColumnResult c = refactor_column<false>(
            pd, pool, a, lu, diag_gmin, check_pivots, rel_threshold, j, buf, lrows, urows,
            [&](int32_t r) { return flag_acquire(done + r); }, rmap);
        if (lane == 0) {
            if (c.timed_out) s_timeout = 1;
            else if (c.code != kStatusOk) atomicMin(&s_fail, fail_key(j, c.code));
            if (c.growth_fail) s_growth = 1;
            flag_release(done + j, 1);
        }
        __syncwarp();
    }
    __syncthreads();
    RefactorResult res;
    if (s_timeout) {
        res.code = kStatusTimeout;
        res.step = -1;
    } else if (s_fail == ~0ull || (amd && !amd_verdict_counts(check_pivots, s_growth != 0))) {
        res.code = kStatusOk;
        res.step = -1;
    } else {
        res.code = static_cast<int32_t>(s_fail & 0xffffffffu);
        res.step = static_cast<int32_t>(s_fail >> 32);
    }
    __syncthreads();
    return res;
}

// x <- A^{-1} x (SparseMatrix::solve, or AmdLuSolver::solve,
// amd_lu_solver.cpp:303-344, for AMD-LU plans) by the whole CTA; w is an
// n-vector of scratch.  Level-synchronous, a thread per row.  Each row
// applies its updates in the order the reference's column-oriented sweeps
// reach it: forward columns ascending; backward ascending for Markowitz
// (row dot product, solve.cpp:30-44), descending for AMD-LU.  Begins and ends
// with __syncthreads().
__device__ inline void cta_solve(const PlanDesc& pd, const int32_t* __restrict__ pool,
                                 const double* __restrict__ lu, double* __restrict__ x,
                                 double* __restrict__ w) {
    const int32_t n = pd.n;
    const bool amd = pd.kind == kPlanAmdLu;
    const int32_t* perm_row = pool + pd.off[PA_perm_row];
    const int32_t* perm_col = pool + pd.off[PA_perm_col];
    const int32_t* diag_pos = pool + pd.off[PA_diag_pos];
    __syncthreads();
    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) w[i] = x[perm_row[i]];
    __syncthreads();
    {   // forward: L with the reciprocal pivot, row-oriented gather
        const int32_t* lp = pool + pd.off[PA_lrow_ptr];
        const int32_t* lpos = pool + pd.off[PA_lrow_pos];
        const int32_t* lcol = pool + pd.off[PA_lrow_col];
        const int32_t* lev_ptr = pool + pd.off[PA_fwd_lev_ptr];
        const int32_t* lev = pool + pd.off[PA_fwd_lev];
        for (int32_t l = 0; l < pd.n_fwd_lev; ++l) {
            for (int32_t k = lev_ptr[l] + threadIdx.x; k < lev_ptr[l + 1]; k += blockDim.x) {
                const int32_t i = lev[k];
                double t = w[i];
                if (amd) {
                    for (int32_t e = lp[i]; e < lp[i + 1]; ++e)
                        t = lu_sub(t, lu_mul(lu[lpos[e]], w[lcol[e]]));
                    w[i] = t;
                    continue;
                }
                for (int32_t e = lp[i]; e < lp[i + 1]; ++e) {
                    const double xc = w[lcol[e]];
                    if (xc != 0.0) t = lu_sub(t, lu_mul(xc, lu[lpos[e]]));
                }
                w[i] = (t != 0.0) ? lu_mul(t, lu[diag_pos[i]]) : t;
            }
            __syncthreads();
        }
    }
    {   // backward: Markowitz unit-diagonal U, row dot products in ascending
        // column order; AMD-LU columns descending, then the pivot division
        const int32_t* up = pool + pd.off[PA_urow_ptr];
        const int32_t* upos = pool + pd.off[PA_urow_pos];
        const int32_t* ucol = pool + pd.off[PA_urow_col];
        const int32_t* lev_ptr = pool + pd.off[PA_bwd_lev_ptr];
        const int32_t* lev = pool + pd.off[PA_bwd_lev];
        for (int32_t l = 0; l < pd.n_bwd_lev; ++l) {
            for (int32_t k = lev_ptr[l] + threadIdx.x; k < lev_ptr[l + 1]; k += blockDim.x) {
                const int32_t i = lev[k];
                double t = w[i];
                if (amd) {
                    for (int32_t e = up[i + 1] - 1; e >= up[i]; --e)
                        t = lu_sub(t, lu_mul(lu[upos[e]], w[ucol[e]]));
                    w[i] = __ddiv_rn(t, lu[diag_pos[i]]);
                    continue;
                }
                for (int32_t e = up[i]; e < up[i + 1]; ++e)
                    t = lu_sub(t, lu_mul(lu[upos[e]], w[ucol[e]]));
                w[i] = t;
            }
            __syncthreads();
        }
    }
    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) x[perm_col[i]] = w[i];
    __syncthreads();
}

// Small instances: the whole LU lives in shared memory and warp 0 alone
// refactors and sweeps it -- no completion flags and no global-memory round
// trips on the dependency chain, which dominate for circuits of a few dozen
// unknowns.  The chain itself is the cost there (a 32-stage inverter chain
// factors as a 32-deep sequence of single columns), so the work is laid out
// to keep it short: every column's A values are scattered by the whole CTA
// before the elimination starts, U entries whose L(:, r) is short are applied
// by lane 0 alone with no warp barrier, and the sweeps run row after row on
// lane 0 in pivot order (a topological order of the triangular solves), so
// no level bookkeeping or barrier sits between dependent rows.  Same
// operations in the same order per entry as cta_refactor_flow /
// cta_solve_flow, so the values are bit-identical.  lu_s: pd.nnz_lu doubles;
// w_s: pd.n.
// Dynamic shared memory of a Newton kernel launch: the LU scratch (flow or
// small path) followed by an optional stage for instance workspaces, capped
// so that two CTAs still fit on an SM.
constexpr size_t kStageCapBytes = 100 * 1024;
__host__ __device__ inline size_t stage_bytes_for(size_t scratch_bytes, long long max_stage) {
    if (scratch_bytes >= kStageCapBytes || max_stage <= 0) return 0;
    const size_t want = static_cast<size_t>(max_stage) * sizeof(double);
    const size_t room = kStageCapBytes - scratch_bytes;
    return want < room ? want : room;
}

__host__ __device__ inline bool small_fits(int n, int nnz_lu, int smem_doubles) {
    return n <= 128 && nnz_lu + n <= smem_doubles;
}

// U entries whose L(:, r) has at most this many rows are applied by lane 0
// alone; longer ones by the whole warp.
constexpr int kSmallSerialRows = 4;

// Refactor into lu_s (and lu, written back at the end).  Begins and ends with
// __syncthreads().
static __device__ __noinline__ RefactorResult cta_refactor_small(
    const PlanDesc& pd, const int32_t* __restrict__ pool, const double* __restrict__ a,
    double* __restrict__ lu, double diag_gmin, int check_pivots, double rel_threshold,
    double* lu_s) {
    const int32_t n = pd.n;
    const int32_t* col_ptr = pool + pd.off[PA_col_ptr];
    const int32_t* diag_pos = pool + pd.off[PA_diag_pos];
    const int32_t* lu_src = pool + pd.off[PA_lu_src];
    const int32_t* upd_dst = pool + pd.off[PA_upd_dst];
    const int32_t map16 = pd.map16;
    const int4* umeta = reinterpret_cast<const int4*>(pool + pd.off[PA_umeta]);
    const bool amd = pd.kind == kPlanAmdLu;
    const int32_t* piv_rank = pool + pd.off[PA_piv_rank];
    const int32_t* gmin_pos = pool + pd.off[PA_gmin_pos];
    const int lane = threadIdx.x & 31;
    __shared__ int32_t s_fail_step, s_fail_code;
    __syncthreads();
    // A values of every column at once (the scatter does not depend on the
    // elimination), then diag_gmin on each column's gmin row.
    for (int32_t t = threadIdx.x; t < pd.nnz_lu; t += blockDim.x) {
        const int32_t src = lu_src[t];
        lu_s[t] = (src >= 0) ? a[src] : 0.0;
    }
    if (diag_gmin != 0.0) {
        __syncthreads();
        for (int32_t j = threadIdx.x; j < n; j += blockDim.x) {
            const int32_t gp = amd ? gmin_pos[j] : diag_pos[j] - col_ptr[j];
            if (gp >= 0) lu_s[col_ptr[j] + gp] = __dadd_rn(lu_s[col_ptr[j] + gp], diag_gmin);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) s_fail_step = INT32_MAX;
    if (threadIdx.x < 32 && n > 0) {
        int32_t fail_step = INT32_MAX, fail_code = kStatusOk;
        bool any_growth = false;
        const bool lane0_pivots = !amd && check_pivots != kCheckNumeric;
        int32_t nc0 = col_ptr[0], nc1 = col_ptr[1], ndp = diag_pos[0];
        for (int32_t j = 0; j < n; ++j) {
            const int32_t c0 = nc0, len = nc1 - nc0, dj = ndp - nc0;
            if (j + 1 < n) {  // the next column's bounds, off the dependency chain
                nc0 = nc1;
                nc1 = col_ptr[j + 2];
                ndp = diag_pos[j + 1];
            }
            double colmax = 0.0;  // AMD-LU: largest |U(r, j)| applied (lane 0)
            for (int32_t q = 0; q < dj; ++q) {
                const int4 m = umeta[c0 + q];  // r, diag_pos[r], |L(:, r)|, upd_start
                if (m.z <= kSmallSerialRows) {
                    if (lane == 0) {
                        const double u = amd ? lu_s[c0 + q] : lu_mul(lu_s[c0 + q], lu_s[m.y]);
                        colmax = fmax(colmax, fabs(u));
                        lu_s[c0 + q] = u;
                        for (int32_t t = 0; t < m.z; ++t) {
                            const int32_t d = c0 + upd_at(upd_dst, map16, m.w + t);
                            lu_s[d] = lu_sub(lu_s[d], lu_mul(u, lu_s[m.y + 1 + t]));
                        }
                    }
                } else {
                    __syncwarp();  // lane 0's serial updates visible to the warp
                    double u = 0.0;
                    if (lane == 0) {
                        u = amd ? lu_s[c0 + q] : lu_mul(lu_s[c0 + q], lu_s[m.y]);
                        colmax = fmax(colmax, fabs(u));
                        lu_s[c0 + q] = u;
                    }
                    u = __shfl_sync(0xffffffffu, u, 0);
                    for (int32_t t = lane; t < m.z; t += 32) {
                        const int32_t d = c0 + upd_at(upd_dst, map16, m.w + t);
                        lu_s[d] = lu_sub(lu_s[d], lu_mul(u, lu_s[m.y + 1 + t]));
                    }
                    __syncwarp();
                }
            }
            int32_t code = kStatusOk;
            if (lane0_pivots) {
                // refactorize(): a zero pivot fails; the reciprocal is stored.
                if (lane == 0) {
                    const double piv = lu_s[c0 + dj];
                    code = (piv == 0.0) ? kStatusSingular : kStatusOk;
                    lu_s[c0 + dj] = __drcp_rn(piv);
                }
            } else {
                __syncwarp();
                const double piv = lu_s[c0 + dj];
                if (amd) {
                    colmax = __shfl_sync(0xffffffffu, colmax, 0);
                    const AmdColumn v = amd_column_status(lu_s + c0, dj, len, colmax,
                                                          check_pivots, piv_rank[j], gmin_pos[j],
                                                          lane);
                    code = v.code;
                    any_growth = any_growth || v.growth_fail;
                    for (int32_t t = dj + 1 + lane; t < len; t += 32)
                        lu_s[c0 + t] = __ddiv_rn(lu_s[c0 + t], piv);
                } else {
                    double largest = 0.0;
                    for (int32_t t = dj + 1 + lane; t < len; t += 32)
                        largest = fmax(largest, fabs(lu_s[c0 + t]));
                    largest = warp_max(largest);
                    code = !(largest * rel_threshold < fabs(piv)) ? kStatusReorder : kStatusOk;
                    __syncwarp();
                    if (lane == 0) lu_s[c0 + dj] = __drcp_rn(piv);
                }
                __syncwarp();
            }
            if (lane == 0 && code != kStatusOk && j < fail_step) {
                fail_step = j;
                fail_code = code;
            }
        }
        if (amd && !amd_verdict_counts(check_pivots, any_growth)) fail_step = INT32_MAX;
        if (lane == 0) {
            s_fail_step = fail_step;
            s_fail_code = fail_code;
        }
    }
    __syncthreads();
    for (int32_t k = threadIdx.x; k < pd.nnz_lu; k += blockDim.x) lu[k] = lu_s[k];
    RefactorResult res;
    res.step = s_fail_step == INT32_MAX ? -1 : s_fail_step;
    res.code = s_fail_step == INT32_MAX ? kStatusOk : s_fail_code;
    __syncthreads();
    return res;
}

// x <- A^{-1} x from the LU in lu_s: lane 0, row after row in pivot order
// (forward: ascending, backward: descending), each row's entries in the
// order of the level-scheduled sweeps.  The next row's bounds and pivot are
// fetched while the current row is computed, so only the values carry the
// dependency from row to row.  Begins and ends with __syncthreads().
static __device__ __noinline__ void cta_solve_small(const PlanDesc& pd,
                                                    const int32_t* __restrict__ pool,
                                                    const double* __restrict__ lu_s,
                                                    double* __restrict__ x,
                                                    double* __restrict__ w) {
    const int32_t n = pd.n;
    const int32_t* perm_row = pool + pd.off[PA_perm_row];
    const int32_t* perm_col = pool + pd.off[PA_perm_col];
    const int32_t* diag_pos = pool + pd.off[PA_diag_pos];
    const bool amd = pd.kind == kPlanAmdLu;
    __syncthreads();
    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) w[i] = x[perm_row[i]];
    __syncthreads();
    if (threadIdx.x == 0 && n > 0) {
        {   // forward: L (Markowitz: skip zero operands, then the reciprocal pivot)
            const int32_t* lp = pool + pd.off[PA_lrow_ptr];
            const int32_t* lpos = pool + pd.off[PA_lrow_pos];
            const int32_t* lcol = pool + pd.off[PA_lrow_col];
            int32_t e = lp[0], e1 = lp[1];
            double piv = amd ? 0.0 : lu_s[diag_pos[0]];
            for (int32_t i = 0; i < n; ++i) {
                const bool more = i + 1 < n;
                const int32_t e1n = more ? lp[i + 2] : 0;
                const double pivn = (more && !amd) ? lu_s[diag_pos[i + 1]] : 0.0;
                double t = w[i];
                if (amd) {
                    for (; e < e1; ++e) t = lu_sub(t, lu_mul(lu_s[lpos[e]], w[lcol[e]]));
                    w[i] = t;
                } else {
                    for (; e < e1; ++e) {
                        const double l = lu_s[lpos[e]];
                        const double xc = w[lcol[e]];
                        if (xc != 0.0) t = lu_sub(t, lu_mul(xc, l));
                    }
                    w[i] = (t != 0.0) ? lu_mul(t, piv) : t;
                }
                e1 = e1n;
                piv = pivn;
            }
        }
        {   // backward: U row dot products (AMD-LU: columns descending, then
            // the pivot division)
            const int32_t* up = pool + pd.off[PA_urow_ptr];
            const int32_t* upos = pool + pd.off[PA_urow_pos];
            const int32_t* ucol = pool + pd.off[PA_urow_col];
            int32_t e0 = up[n - 1], e1 = up[n];
            double piv = amd ? lu_s[diag_pos[n - 1]] : 0.0;
            for (int32_t i = n - 1; i >= 0; --i) {
                const bool more = i > 0;
                const int32_t e0n = more ? up[i - 1] : 0;
                const double pivn = (more && amd) ? lu_s[diag_pos[i - 1]] : 0.0;
                double t = w[i];
                if (amd) {
                    for (int32_t e = e1 - 1; e >= e0; --e)
                        t = lu_sub(t, lu_mul(lu_s[upos[e]], w[ucol[e]]));
                    w[i] = __ddiv_rn(t, piv);
                } else {
                    for (int32_t e = e0; e < e1; ++e)
                        t = lu_sub(t, lu_mul(lu_s[upos[e]], w[ucol[e]]));
                    w[i] = t;
                }
                e1 = e0;
                e0 = e0n;
                piv = pivn;
            }
        }
    }
    __syncthreads();
    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) x[perm_col[i]] = w[i];
    __syncthreads();
}

// Entries of a row the dataflow sweeps fetch ahead of their waits.
constexpr int kSweepChunk = 8;

// Shared memory of the dataflow solve: the n-vector and n completion flags.
__host__ __device__ inline size_t flow_solve_smem_bytes(int n) {
    return (sizeof(double) + sizeof(int32_t)) * static_cast<size_t>(n);
}

// Wait (bounded) until flag[i] is set; returns false on timeout.  The flag is
// read with acquire semantics, so the value read after it is the one the
// producer wrote before its release store.
__device__ __forceinline__ bool wait_flag(volatile int32_t* flag, int32_t i) {
    if (flag_acquire(flag + i) != 0) return true;
    const int limit = c_wait_limit;
    int spins = 0;
    while (flag_acquire(flag + i) == 0) {
        if (++spins > limit) return false;
        __nanosleep(32);
    }
    return true;
}

// x <- A^{-1} x (SparseMatrix::solve) by the whole CTA, dataflow schedule:
// thread t takes rows t, t + blockDim, ... of the level-sorted order and
// waits, entry by entry, for the rows it reads.  The vector and the flags live
// in shared memory (flow_solve_smem_bytes); L and U are read from the
// row-major copies the refactor wrote.  Same arithmetic, in the same order
// per row, as cta_solve.  Returns false if a bounded wait gave up.
static __device__ __noinline__ bool cta_solve_flow(const PlanDesc& pd, const int32_t* __restrict__ pool,
                                      const double* __restrict__ lu,
                                      const double* __restrict__ lrows,
                                      const double* __restrict__ urows, double* __restrict__ x,
                                      double* smem) {
    const int32_t n = pd.n;
    const int32_t* perm_row = pool + pd.off[PA_perm_row];
    const int32_t* perm_col = pool + pd.off[PA_perm_col];
    const int32_t* diag_pos = pool + pd.off[PA_diag_pos];
    const bool amd = pd.kind == kPlanAmdLu;
    volatile double* w = smem;
    volatile int32_t* done = reinterpret_cast<volatile int32_t*>(smem + n);
    __shared__ int32_t s_ok;
    __syncthreads();
    if (threadIdx.x == 0) s_ok = 1;
    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) {
        w[i] = x[perm_row[i]];
        done[i] = 0;
    }
    __syncthreads();
    bool ok = true;
    {   // forward: L with the reciprocal pivot
        const int32_t* lp = pool + pd.off[PA_lrow_ptr];
        const int32_t* lcol = pool + pd.off[PA_lrow_col];
        const int32_t* order = pool + pd.off[PA_fwd_lev];
        for (int32_t k = threadIdx.x; k < n; k += blockDim.x) {
            const int32_t i = order[k];
            double t = w[i];
            const int32_t e1 = lp[i + 1];
            // The row's entries are fetched kSweepChunk at a time ahead of
            // the waits, so a row pays one memory round trip per chunk, not
            // one per entry; they are still applied one by one in order.
            for (int32_t e0 = lp[i]; e0 < e1; e0 += kSweepChunk) {
                int32_t cs[kSweepChunk];
                double vs[kSweepChunk];
#pragma unroll
                for (int u = 0; u < kSweepChunk; ++u) {
                    cs[u] = (e0 + u < e1) ? lcol[e0 + u] : 0;
                    vs[u] = (e0 + u < e1) ? lrows[e0 + u] : 0.0;
                }
#pragma unroll
                for (int u = 0; u < kSweepChunk; ++u) {
                    if (e0 + u >= e1) break;
                    const int32_t c = cs[u];
                    if (ok && !wait_flag(done, c)) ok = false;
                    const double xc = w[c];
                    if (amd) t = lu_sub(t, lu_mul(vs[u], xc));
                    else if (xc != 0.0) t = lu_sub(t, lu_mul(xc, vs[u]));
                }
            }
            if (!amd) t = (t != 0.0) ? lu_mul(t, lu[diag_pos[i]]) : t;
            w[i] = t;
            flag_release(done + i, 1);
        }
    }
    __syncthreads();
    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) done[i] = 0;
    __syncthreads();
    {   // backward: Markowitz unit-diagonal U, columns ascending; AMD-LU
        // columns descending, then the pivot division
        const int32_t* up = pool + pd.off[PA_urow_ptr];
        const int32_t* ucol = pool + pd.off[PA_urow_col];
        const int32_t* order = pool + pd.off[PA_bwd_lev];
        for (int32_t k = threadIdx.x; k < n; k += blockDim.x) {
            const int32_t i = order[k];
            double t = w[i];
            const int32_t e0 = up[i], e1 = up[i + 1];
            const int32_t len = e1 - e0;
            for (int32_t m0 = 0; m0 < len; m0 += kSweepChunk) {
                int32_t cs[kSweepChunk];
                double vs[kSweepChunk];
#pragma unroll
                for (int u = 0; u < kSweepChunk; ++u) {
                    const int32_t e = amd ? e1 - 1 - (m0 + u) : e0 + m0 + u;
                    cs[u] = (m0 + u < len) ? ucol[e] : 0;
                    vs[u] = (m0 + u < len) ? urows[e] : 0.0;
                }
#pragma unroll
                for (int u = 0; u < kSweepChunk; ++u) {
                    if (m0 + u >= len) break;
                    const int32_t c = cs[u];
                    if (ok && !wait_flag(done, c)) ok = false;
                    t = lu_sub(t, lu_mul(vs[u], w[c]));
                }
            }
            w[i] = amd ? __ddiv_rn(t, lu[diag_pos[i]]) : t;
            flag_release(done + i, 1);
        }
    }
    if (!ok) s_ok = 0;
    __syncthreads();
    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) x[perm_col[i]] = w[i];
    const bool all_ok = (s_ok != 0);
    __syncthreads();
    return all_ok;
}

// x <- A^{-T} x (SparseMatrix::solve_transposed) by the whole CTA.  AMD-LU
// plans (the reference's AmdLuSolver has no transposed solve) use
// A^T = Q U^T L^T P: U^T forward with the pivot division, then unit L^T.
__device__ inline void cta_solve_transposed(const PlanDesc& pd, const int32_t* __restrict__ pool,
                                            const double* __restrict__ lu, double* __restrict__ x,
                                            double* __restrict__ w) {
    const int32_t n = pd.n;
    const int32_t* perm_row = pool + pd.off[PA_perm_row];
    const int32_t* perm_col = pool + pd.off[PA_perm_col];
    const int32_t* col_ptr = pool + pd.off[PA_col_ptr];
    const int32_t* row_idx = pool + pd.off[PA_row_idx];
    const int32_t* diag_pos = pool + pd.off[PA_diag_pos];
    const bool amd = pd.kind == kPlanAmdLu;
    __syncthreads();
    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) w[i] = x[perm_col[i]];
    __syncthreads();
    {   // forward over U^T: column c gathers its U entries in stored order
        // (AMD-LU: then divides by the pivot)
        const int32_t* lev_ptr = pool + pd.off[PA_col_lev_ptr];
        const int32_t* lev = pool + pd.off[PA_col_lev];
        for (int32_t l = 0; l < pd.n_col_lev; ++l) {
            for (int32_t k = lev_ptr[l] + threadIdx.x; k < lev_ptr[l + 1]; k += blockDim.x) {
                const int32_t c = lev[k];
                double t = w[c];
                for (int32_t q = col_ptr[c]; q < diag_pos[c]; ++q) {
                    const double xr = w[row_idx[q]];
                    if (xr != 0.0) t = lu_sub(t, lu_mul(xr, lu[q]));
                }
                w[c] = amd ? __ddiv_rn(t, lu[diag_pos[c]]) : t;
            }
            __syncthreads();
        }
    }
    {   // backward over L^T (Markowitz: then the reciprocal pivot)
        const int32_t* lev_ptr = pool + pd.off[PA_tbw_lev_ptr];
        const int32_t* lev = pool + pd.off[PA_tbw_lev];
        for (int32_t l = 0; l < pd.n_tbw_lev; ++l) {
            for (int32_t k = lev_ptr[l] + threadIdx.x; k < lev_ptr[l + 1]; k += blockDim.x) {
                const int32_t i = lev[k];
                double t = w[i];
                for (int32_t q = diag_pos[i] + 1; q < col_ptr[i + 1]; ++q)
                    t = lu_sub(t, lu_mul(lu[q], w[row_idx[q]]));
                w[i] = amd ? t : lu_mul(t, lu[diag_pos[i]]);
            }
            __syncthreads();
        }
    }
    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) x[perm_row[i]] = w[i];
    __syncthreads();
}

}  // namespace nsg
