// Device descriptors of the batched DC Newton kernel.
#pragma once
#include "lu_device.cuh"

#include <cstdint>

namespace nsg {

// Stamp-program arrays of one circuit in the program pool.
enum DcProgArray : int {
    DP_slot_ptr, DP_slot_terms, DP_rhs_ptr, DP_rhs_terms, DP_ucb_ptr, DP_ucb_terms,
    DP_term_op, DP_term_param, DP_diodes, DP_caps, DP_srcs, DP_mos, DP_grad, DP_COUNT
};

struct DcDesc {
    int32_t index;       // the instance's position in the caller's arrays
    int32_t plan;        // PlanDesc index (LU structure)
    int32_t n;           // unknowns
    int32_t num_nodes;   // node unknowns come first, branch currents after
    int32_t nnz;         // matrix slots
    int32_t n_const;     // constant terms
    int32_t n_diodes;
    int32_t n_caps;
    int32_t n_srcs;      // waveform sources
    int32_t n_mos;       // MOSFETs (level 1)
    int32_t n_grad;      // gradient-program records (DC adjoint)
    int32_t n_states;    // per state vector (2 per capacitor, 17 per MOSFET)
    int64_t prog_off[DP_COUNT];  // int32-word offsets into the program pool
    int64_t param_off;           // into the caller's parameter array
    int64_t sol_off;             // into the caller's solution array
    // workspace (doubles): solution, previous iterate, sweep scratch, matrix
    // values, LU values, term values, diode constants
    int64_t x_off, xold_off, w_off, a_off, lu_off, tv_off, dconst_off;
    int64_t lrows_off, urows_off;  // row-major copies of L and U for the sweeps
    int64_t state_off;             // four state vectors of n_states doubles
    int64_t mrec_off;              // per-MOSFET persistent load values
    int64_t dcsave_off;            // gmin-stepping save area (x, state0..2)
    // Doubles from x_off on that a launch may stage in shared memory (every
    // per-iteration region: vectors, matrix, LU, terms, states, history).
    int64_t stage_len;
};

// SimOptions of the reference (src/core/types.hpp:24-66) used by the loop.
struct NewtonOptions {
    double reltol;
    double vntol;
    double abstol;
    double gmin;       // device gmin and dead-node pin
    double diag_gmin;  // solver diagonal regularisation
    int32_t max_iter;  // itl1
    int32_t first_aid; // where the operating-point cascade starts: kAidDirect (0),
                       // kAidSource (source stepping), kAidGain (gain stepping),
                       // kAidPseudoTransient
    double src_fact = 1.0;  // independent-source scale (SimOptions::src_fact)
    int32_t want_residual = 0;  // report NewtonResult::residual (pseudo-transient)
    int32_t pad = 0;
};

enum : int32_t { kAidDirect = 0, kAidSource = 1, kAidGain = 2, kAidPseudoTransient = 3 };

constexpr int kDiodeTermCount = 5;
constexpr int kCapTermCount = 4;
constexpr int kSrcTermCount = 2;
constexpr int kMosTermCount = 26;
constexpr int kMosRecCount = 12;
// MOSFET table: (d, g, s, b, param, state, family) per device; family 0
// level-1 (kernels/mos1_model.cuh), 1 BSIM4v7 (kernels/bsim4_model.cuh).
constexpr int kMosTabStride = 7;
constexpr int kMosFamilyBsim4 = 1;
// CONSTKoverQ * 300.15 evaluated as the reference's diode temperature code does.
constexpr double kKoverQTimesTnom = (1.38064852e-23 / 1.6021766208e-19) * 300.15;

// Integrator context of one instance (IntegratorCtx, src/core/types.hpp:73-94),
// written by thread 0, read by every thread after a barrier.
struct IntegCtx {
    double ag[3];
    double xmu_ratio;
    double delta;
    double delta_old[3];
    double time;      // source time (update_source_time)
    int32_t mode;
    int32_t order;
    int32_t method;   // 0 trapezoidal, 1 Gear
    int32_t pad;
};

// Solver state of one instance across newton() calls (NeoSolver's flag).
struct SolverState {
    int32_t factored;  // a numeric() has succeeded on this plan
};

// Operating-point phases (kernels/dc_op.cuh): the direct attempt, true gmin
// stepping and its final solve, diagonal gmin stepping and its final solve,
// then source (or gain) stepping: the solve at zero sources, its diagonal
// gmin ramp, the ramp of the source fraction.
enum DcOpPhase : int32_t {
    kOpDirect = 0,
    kOpTrueGmin = 1,
    kOpTrueGminFinal = 2,
    kOpDiagGmin = 3,
    kOpDiagGminFinal = 4,
    kOpDone = 5,
    kOpSrcFirst = 6,
    kOpSrcZeroGmin = 7,
    kOpSrcStep = 8,
    kOpPtc = 9,        // pseudo-transient: a step at diag_gmin = C/dt
    kOpPtcProbe = 10,  // the probe solve at the target diag_gmin
    kOpPtcFinal = 11,  // the final attempt after the step loop
};

// Operating-point controller of one instance, kept in global memory across
// launches (zeroed by the host before a fresh run).
struct DcCtl {
    int32_t phase, total, code, ctx_mode;  // ctx_mode: mode of the next Newton call
    int32_t active, r_iter, r_mode, r_devconv;  // Newton resume record
    int32_t action, solves, method, pad;  // method: ConvergenceMethod of the result
    double cur, factor, old, numeric_diag_gmin;  // stepping gmin, factor, OldGmin; diag_gmin of a stopped numeric()
    // source / gain stepping: accepted fraction, step, fraction under
    // solve, diag_gmin of the zero-source ramp; ramp index, the failed first
    // solve's iterations, 1 for gain stepping (sources unscaled)
    double frac, step, next, zdiag;
    int32_t zi, r0_iters, gain, pad2;
    // pseudo-transient: pseudo timestep, previous residual (-1: none), the
    // probe threshold on C/dt; step index
    double ptc_dt, ptc_prev, ptc_probe;
    int32_t ptc_k, pad3;
};

enum : int32_t { kActNone = 0, kActZeroSave = 1, kActSave = 2, kActRestore = 3 };

// Per-instance DC status.
enum : int32_t {
    kDcConverged = 0,
    kDcNoConvergence = 1,  // itl1 iterations without convergence
    // kStatusSingular (102), kStatusReorder (103), kStatusTimeout (104)
};

}  // namespace nsg
