// Device descriptors of the batched transient kernel.
#pragma once
#include "dc_device.cuh"

#include <cstdint>

namespace nsg {

struct TranDesc {
    int32_t tran_plan;  // PlanDesc of the transient solver (ordered on the first step's matrix)
    int32_t n_bps;      // source breakpoints of this instance
    int64_t bp_off;     // into the breakpoint array
    int64_t out_off;    // first output point slot of this instance
    int64_t hist_off;   // workspace: three history vectors of n doubles
    double dt0;         // initial timestep (transient.cpp:851-865)
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

// Per-instance transient status.
enum : int32_t {
    kTranOk = 0,
    kTranDcFailed = 2,      // the initial operating point did not converge
    kTranNewtonFailed = 3,  // Newton failed at the minimum timestep
    kTranTooManySteps = 4,  // kMaxTransientIterations reached
    // kStatusReorder (103), kStatusTimeout (104)
};

}  // namespace nsg
