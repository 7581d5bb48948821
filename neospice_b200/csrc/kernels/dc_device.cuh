// Device descriptors of the batched DC Newton kernel.
#pragma once
#include "lu_device.cuh"

#include <cstdint>

namespace nsg {

// Stamp-program arrays of one circuit in the program pool.
enum DcProgArray : int {
    DP_slot_ptr, DP_slot_terms, DP_rhs_ptr, DP_rhs_terms, DP_ucb_ptr, DP_ucb_terms,
    DP_term_op, DP_term_param, DP_diodes, DP_caps, DP_srcs, DP_COUNT
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
    int32_t n_states;    // per state vector (2 per capacitor)
    int64_t prog_off[DP_COUNT];  // int32-word offsets into the program pool
    int64_t param_off;           // into the caller's parameter array
    int64_t sol_off;             // into the caller's solution array
    // workspace (doubles): solution, previous iterate, sweep scratch, matrix
    // values, LU values, term values, diode state, diode constants
    int64_t x_off, xold_off, w_off, a_off, lu_off, tv_off, dstate_off, dconst_off;
    int64_t lrows_off, urows_off;  // row-major copies of L and U for the sweeps
    int64_t state_off;             // four state vectors of n_states doubles
};

// SimOptions of the reference (src/core/types.hpp:24-66) used by the loop.
struct NewtonOptions {
    double reltol;
    double vntol;
    double abstol;
    double gmin;       // device gmin and dead-node pin
    double diag_gmin;  // solver diagonal regularisation
    int32_t max_iter;  // itl1
    int32_t pad;
};

constexpr int kDiodeTermCount = 5;
constexpr int kCapTermCount = 4;
constexpr int kSrcTermCount = 2;
// CONSTKoverQ * 300.15 evaluated as the reference's diode temperature code does.
constexpr double kKoverQTimesTnom = (1.38064852e-23 / 1.6021766208e-19) * 300.15;

// Per-instance DC status.
enum : int32_t {
    kDcConverged = 0,
    kDcNoConvergence = 1,  // itl1 iterations without convergence
    // kStatusSingular (102), kStatusReorder (103), kStatusTimeout (104)
};

}  // namespace nsg
