// Device descriptors of the batched transient kernel.
#pragma once
#include "dc_device.cuh"

#include <cstdint>

namespace nsg {

struct TranDesc {
    int32_t tran_plan;  // PlanDesc of the transient solver (ordered by the host on the
                        // first transient iteration's matrix; -1 until then)
    int32_t n_bps;      // source breakpoints of this instance
    int64_t bp_off;     // into the breakpoint array
    int64_t out_off;    // first output point slot of this instance
    int64_t hist_off;   // workspace: three history vectors of n doubles
    double dt0;         // initial timestep (transient.cpp:851-865)
    int64_t x0_off;     // recording: the operating point (n doubles) in the x0 record
};

// Integration record of one accepted timepoint (recording on): what the
// adjoint needs to replay the step with the same formula.
struct StepRecord {
    double ag[3];       // NIintegrate coefficients
    double xmu_ratio;   // trapezoidal: weight of the previous current
    int32_t order, method, pad[2];
};

// SimOptions / .tran parameters of the transient driver.
struct TranOptions {
    NewtonOptions nopt;   // reltol, vntol, abstol, gmin, diag_gmin, max_iter (DC preamble)
    double tstep, tstop;
    double dt_min, dt_max;
    double trtol, chgtol, xmu, restart_scale;
    int32_t itl4;
    int32_t use_gear;
    int32_t max_points;   // output capacity per instance
    int32_t nprobe;       // unknowns stored per output point
};

enum TranPhase : int32_t { kTrInit = 0, kTrDc = 1, kTrPrepare = 2, kTrStep = 3, kTrDone = 4 };

// Everything one instance's transient carries between launches (global
// memory, zeroed by the host before a fresh run; a launch works on a copy in
// shared memory and writes it back when it stops).
struct TranCtl {
    DcCtl dc;               // the operating point's controller
    IntegCtx ctx;           // integrator context
    double time, dt, prev_dt, prev_prev_dt, saved_delta, proposed_dt, device_dt;
    double need_diag_gmin;  // diag_gmin of the numeric() the host must redo
    int32_t phase, status, step_mode, need;
    int32_t order, step_count, steps_after_bp, order_cooldown;
    int32_t ringing_cooldown, rejected, total_iterations, newton_iters;
    int32_t bp_head, points, tried_delmin, crossed_src_bp;
    SolverState dc_solver, tr_solver;  // the DC and the transient solver
    int32_t ringing, need_plan;        // need_plan: 0 DC, 1 transient
    int32_t nr_active, nr_iter, nr_mode, nr_devconv;  // transient Newton resume record
    int32_t hist[3], pad0;
    int32_t stperm[4];      // buffer of state0..state3 in the ring
};

// What the launch needs to size one CTA: the batch's largest LU column and
// unknown count (dataflow scratch), largest staged workspace, largest
// small-path LU (nnz_lu + n doubles), largest plan (int32 words) and most
// devices of one family in one instance (the device loads' parallelism).
struct TranShape {
    int32_t max_col, max_n;
    int64_t max_stage;
    int32_t max_small_lu;
    int64_t max_plan_words;
    int32_t max_devices;
    int32_t force_threads;   // nsg_tran_batch_set_shape (0: automatic)
    int32_t force_blocks;
};

// Per-instance transient status.
enum : int32_t {
    kTranOk = 0,
    kTranDcFailed = 2,      // the initial operating point did not converge
    kTranNewtonFailed = 3,  // Newton failed at the minimum timestep
    kTranTooManySteps = 4,  // kMaxTransientIterations reached
    // kStatusReorder (103), kStatusTimeout (104), kStatusNeedOrder (105):
    // 103 / 105 stop the instance for the host, which (re-)orders and resumes it
};

}  // namespace nsg
