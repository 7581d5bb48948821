/*
 * nsgpu — B200 (sm_100a) batched FP64 sparse refactor and triangular solves
 * for the neospice Newton inner loop, behind a plain C ABI.
 *
 * Conventions
 *   - Every entry point returns an int status: NSG_OK, or an NSG_ERR_* code
 *     with a message available from nsg_last_error() (per thread).  No C++
 *     exception crosses this boundary.
 *   - Pointers named d_* are device pointers (cudaMalloc / torch CUDA
 *     memory) on the current device; `stream` is a cudaStream_t (may be 0).
 *     All other pointers are host memory.
 *   - Matrices are given in the caller's CSC pattern (0-based, rows
 *     ascending within a column), exactly the slot order of the reference's
 *     SparsityPattern / NumericMatrix (src/core/matrix.hpp:16-93).
 *   - Per-instance status codes mirror SparseError (src/solver/error.hpp:5-13):
 *     0 OK, 102 singular (zero pivot), plus 103 when a re-validated pivot
 *     fails the relative threshold and the instance needs a host re-order.
 */
#ifndef NSGPU_H
#define NSGPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define NSG_OK 0
#define NSG_ERR_INVALID 1    /* bad argument or misuse (reference: std::logic_error / invalid_argument) */
#define NSG_ERR_CUDA 2       /* a CUDA runtime call failed */
#define NSG_ERR_NOMEM 8      /* SparseError::NoMemory */
#define NSG_SINGULAR 102     /* SparseError::Singular / ZeroDiag */
#define NSG_REORDER 103      /* pivot failed re-validation: run nsg_topology_numeric */
#define NSG_TIMEOUT 104      /* a bounded dependency wait on the GPU gave up; no result */

typedef struct nsg_topology nsg_topology;
typedef struct nsg_batch nsg_batch;

/* Message of the last failing call on this thread ("" if none). */
const char* nsg_last_error(void);

/* Polls a dependency wait inside the dataflow and grid-wide kernels makes
 * before it gives up; the instance then reports NSG_TIMEOUT (104) and the
 * kernel still runs to its end, so the context stays usable.  Default 2^22
 * polls (seconds; a wait that runs out means a broken schedule, not a slow
 * one).  0 gives up at the first wait that has to poll -- used by tests to
 * exercise the give-up path.  Applies to every kernel of the library on the
 * current device.  No counterpart in the reference (its factor runs on one
 * thread and never waits). */
int nsg_set_wait_limit(int polls);

/* ---- Symbolic phase (host) ------------------------------------------------
 * nsg_topology_order: NeoSolver::symbolic followed by the first
 * NeoSolver::numeric (src/core/neo_solver.cpp:184-245): load values, MNA
 * pre-order, add diag_gmin, Markowitz order_and_factor with relThr 1e-3,
 * absThr 1e-13 and diagonal pivoting (src/solver/factor.cpp:911-978).  The
 * pivot sequence and fill pattern are bit-identical to the reference's.
 * Returns NSG_SINGULAR (and no topology) when the reference would report a
 * singular matrix. */
int nsg_topology_order(int n, int nnz, const int* col_ptr, const int* row_idx,
                       const double* values, double diag_gmin, nsg_topology** out);

/* Factorization engines (make_solver, src/core/make_solver.cpp:156-178).
 *   NSG_SOLVER_MARKOWITZ  NeoSolver: Sparse-1.3 Markowitz ordering.
 *   NSG_SOLVER_AMDLU      AmdLuSolver (src/core/amd_lu_solver.cpp:11-358):
 *                         AMD column order, left-looking LU with threshold
 *                         partial pivoting, fixed-pivot replay refactor.
 *   NSG_SOLVER_AUTO_AMDLU AutoFallbackSolver (make_solver.cpp:71-145): AMD-LU,
 *                         switching to Markowitz for good when the first
 *                         factorization is singular. */
#define NSG_SOLVER_MARKOWITZ 0
#define NSG_SOLVER_AMDLU 1
#define NSG_SOLVER_AUTO_AMDLU 2

/* make_solver(num_vars, is_linear)'s choice: NEOSPICE_SOLVER=amdlu|klu or
 * markowitz|sparse, else NEOSPICE_FORCE_AMDLU (non-empty, not "0"), else
 * NSG_SOLVER_AUTO_AMDLU for linear circuits of at least 256 unknowns and
 * NSG_SOLVER_MARKOWITZ otherwise (make_solver.cpp:41-55, 166-174). */
int nsg_solver_select(int num_vars, int is_linear);

/* nsg_topology_order with an explicit engine: for the AMD-LU engines,
 * AmdLuSolver::symbolic then numeric (amd_lu_solver.cpp:11-38, 74-197,
 * 273-278); the pivot sequence, fill and replay order are the reference's.
 * Device values of an AMD-LU topology follow AmdLuSolver's layout: U
 * unscaled, L divided by the pivot, pivots stored as is. */
int nsg_topology_order_solver(int n, int nnz, const int* col_ptr, const int* row_idx,
                              const double* values, double diag_gmin, int solver,
                              nsg_topology** out);

/* Engine of a topology's current plan (NSG_SOLVER_MARKOWITZ or
 * NSG_SOLVER_AMDLU; an auto topology reports the engine it settled on), or
 * NSG_ERR_INVALID. */
int nsg_topology_solver(const nsg_topology* topo);

/* amd_ordering (src/core/amd.cpp:14-143) of a CSC pattern: perm[k] = the
 * original column eliminated at step k (n ints). */
int nsg_amd_order(int n, const int* col_ptr, const int* row_idx, int* perm);

/* nsg_topology_numeric: a later NeoSolver::numeric on the same topology
 * (neo_solver.cpp:219-245): re-validate every pivot on the new values and
 * re-order from the first failing step, as SparseMatrix::order_and_factor
 * does (factor.cpp:929-947).  *reordered is set to the first re-ordered step
 * (1-based) or 0.  Instances sharing this topology in an existing batch must
 * be rebuilt when *reordered != 0. */
int nsg_topology_numeric(nsg_topology* topo, const double* values, double diag_gmin,
                         int* reordered);

/* nsg_topology_import: take a symbolic result computed by the reference's
 * own NeoSolver (the state behind element_ptrs_ after order_and_factor,
 * neo_solver.cpp:113-146): 1-based int_to_ext_row/col of length n, n_elem
 * elements listed column by column in pivot order with 1-based internal
 * rows (ascending) and columns, and for each of the nnz caller slots its
 * element index. */
int nsg_topology_import(int n, int nnz, const int* int_to_ext_row,
                        const int* int_to_ext_col, int n_elem, const int* elem_row,
                        const int* elem_col, const int* slot_to_elem, nsg_topology** out);

/* Sizes: n, caller nnz, LU entries, multiply-subtract updates per refactor,
 * and the level counts of the refactor / forward / backward schedules. */
int nsg_topology_info(const nsg_topology* topo, int* n, int* nnz, int* nnz_lu,
                      long long* updates, int* col_levels, int* fwd_levels,
                      int* bwd_levels);

/* Export in the format nsg_topology_import takes (arrays sized n, n, nnz_lu,
 * nnz_lu, nnz). */
int nsg_topology_export(const nsg_topology* topo, int* int_to_ext_row,
                        int* int_to_ext_col, int* elem_row, int* elem_col,
                        int* slot_to_elem);

/* NeoSolver::numeric_complex (src/core/neo_solver.cpp:228-245): the
 * symbolic phase on complex values ax (2*nnz doubles, (re, im) per CSC slot):
 * MNA pre-order and Markowitz order_and_factor with magnitudes |re| + |im|
 * and complex eliminations (src/solver/factor.cpp:769-806), pivot sequence
 * bit-identical to the reference's.  The AC sweep's first frequency point
 * (src/core/ac.cpp:205-209).  Returns NSG_SINGULAR (and no topology) on a
 * singular matrix, which the reference does not report. */
int nsg_topology_order_complex(int n, int nnz, const int* col_ptr, const int* row_idx,
                               const double* ax, nsg_topology** out);

void nsg_topology_free(nsg_topology* topo);

/* ---- Batches (device) -----------------------------------------------------
 * A batch holds `count` instances, instance i using topos[i] (instances may
 * share a topology).  It owns the device plan and the LU values.  The
 * caller's value and vector arrays are packed instance after instance; the
 * offsets (count+1 entries each, in doubles) come from nsg_batch_layout. */
int nsg_batch_create(int count, nsg_topology* const* topos, nsg_batch** out);
void nsg_batch_free(nsg_batch* batch);
int nsg_batch_layout(const nsg_batch* batch, long long* value_offsets,
                     long long* vector_offsets, long long* lu_offsets);

/* spFactor for every instance: SparseMatrix::factor after load_real and
 * add_diag_gmin (neo_solver.cpp:247-265, factor.cpp:980-1052), with the
 * fixed pivots.  check_pivots != 0 instead applies the re-validation test of
 * a later NeoSolver::numeric (factor.cpp:929-947) and reports NSG_REORDER.
 * AMD-LU topologies: AmdLuSolver::refactorize's replay
 * (amd_lu_solver.cpp:214-271).  Where its pivot-growth test fails the
 * reference re-factors the same values with factor_; the kernel checks
 * whether factor_'s threshold pivoting would choose the plan's pivots (then
 * the replayed values are factor_'s, bit for bit) and reports NSG_REORDER
 * otherwise (run nsg_topology_numeric).  With check_pivots != 0, a numeric():
 * NSG_REORDER unless factor_ would choose the same pivots on these values.
 * d_status[i] / d_fail_step[i] (device int arrays, fail_step optional)
 * receive the per-instance code and the failing 0-based pivot step. */
int nsg_batch_refactor(nsg_batch* batch, const double* d_values, double diag_gmin,
                       int check_pivots, int* d_status, int* d_fail_step, void* stream);

/* Refactor schedule: 0 (default) = dataflow (warps claim columns in pivot
 * order and wait on per-column completion flags, column staged in shared
 * memory; used when the batch's columns fit), 1 = level-synchronous, both
 * one CTA per instance; 2 = grid-wide (instances one after another, each
 * refactored and swept by every SM, for a few large topologies).  All
 * produce bit-identical values. */
int nsg_batch_set_schedule(nsg_batch* batch, int schedule);
/* Shared column buffer per warp of the grid-wide refactor (schedule 2):
 * 1024, 2048 or 4096 doubles, or 0 (default) for the smallest that holds the
 * longest column.  Longer columns are eliminated in place in global memory.
 * No counterpart in the reference (a tuning knob of this schedule). */
int nsg_batch_set_grid_buffer(nsg_batch* batch, int doubles);
/* Columns of an AMD-LU instance the grid-wide refactor (schedule 2, with a
 * 2048- or 4096-double column buffer) hands to whole CTAs instead of single
 * warps: the last `columns` columns, 0 for none, or -1 (default) for the
 * longest suffix of columns that each apply at least 128 updates (the top
 * separators).  Same values either way.  No counterpart in the reference
 * (a tuning knob of this schedule). */
int nsg_batch_set_grid_tail(nsg_batch* batch, int columns);
/* Largest refactor update map (int32 words, one per multiply-subtract) a
 * topology ordered from now on may carry; default 2^30 (4 GiB).  A larger
 * factorization gets no map: its batches run only the grid-wide schedule,
 * which finds each update's destination through a per-warp row -> position
 * map (n words per warp of the grid), and circuit batches refuse it.  No
 * counterpart in the reference (its refactor walks linked lists). */
int nsg_set_update_map_limit(long long words);

/* Schedule autotuner: refactor d_values (as a refactorize()) and solve d_x
 * under each schedule (0 dataflow, 1 level-synchronous, 2 grid-wide), reps
 * times each, time them with CUDA events and keep the fastest.  times_ms[3]
 * (optional) receives the mean refactor+solve time per schedule (-1 if it
 * did not run), *chosen the schedule kept.  d_x is left as given; the
 * factors are those of the last schedule timed (all schedules give
 * bit-identical values).  Allocates temporary device memory. */
int nsg_batch_autotune(nsg_batch* batch, const double* d_values, double* d_x, int reps,
                       float* times_ms, int* chosen, void* stream);

/* spSolve: d_x holds b on entry and x on return, per instance
 * (SparseMatrix::solve, src/solver/solve.cpp:6-47; NeoSolver::solve). */
int nsg_batch_solve(nsg_batch* batch, double* d_x, void* stream);

/* spSolveTransposed: A^T x = b on the same factors
 * (SparseMatrix::solve_transposed, src/solver/solve.cpp:102-141). */
int nsg_batch_solve_transposed(nsg_batch* batch, double* d_x, void* stream);

/* Allocation-free solve.  No counterpart in the reference: it exists for
 * callers that must not allocate device memory when they solve -- a simulator
 * held to a fixed memory budget, code running inside another framework's
 * memory pool, or a latency-critical loop that cannot afford the implicit
 * synchronisation of cudaMalloc/cudaFree.  Same result as nsg_batch_solve
 * (bit for bit), but the per-instance sweep workspace comes from a fixed
 * array of NSG_STATIC_SCRATCH_DOUBLES doubles (8 MiB) compiled into the
 * library, which every GPU that loads the library keeps until the process
 * exits; the call itself allocates nothing.
 *   - Batches whose unknowns total more than NSG_STATIC_SCRATCH_DOUBLES are
 *     rejected with NSG_ERR_INVALID (see nsg_last_error).
 *   - Call it with the batch's device current (the device that was current
 *     at nsg_batch_create); another current device gives NSG_ERR_INVALID.
 *   - The first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress) with that device current and keeps it; make that
 *     first call before any stream capture.  Resetting that device
 *     (cudaDeviceReset) afterwards is not supported: the kept address would
 *     no longer be the array's.
 *   - All calls share the one array: calls that overlap on the GPU (different
 *     streams, or different batches at once) race.  The array keeps the last
 *     call's contents; nothing in it has to start at zero. */
#define NSG_STATIC_SCRATCH_DOUBLES (1LL << 20)
int nsg_batch_solve_static_scratch(nsg_batch* batch, double* d_x, void* stream);

/* Batched AC: SparseMatrix::factor_complex (refactorize_complex,
 * src/solver/factor.cpp:1054-1141) of every instance with the plan's fixed
 * pivots.  d_ax: complex values interleaved (re, im), 2*value_offsets per
 * instance (nsg_batch_layout); d_lu: caller-owned device buffer of
 * 2*lu_offsets[count] doubles receiving the factors (same positions as the
 * real LU, interleaved); d_status per instance: 0, 102 (zero pivot) or 104.
 * Markowitz plans only (the reference's AC uses NeoSolver). */
int nsg_batch_refactor_complex(nsg_batch* batch, const double* d_ax, double* d_lu, int* d_status,
                               void* stream);
/* SparseMatrix::solve_complex (src/solver/solve.cpp:49-100) on d_lu: d_x
 * holds b on entry and x on return, interleaved, 2*vector_offsets per
 * instance.  The first call allocates the batch's complex sweep workspace. */
int nsg_batch_solve_complex(nsg_batch* batch, const double* d_lu, double* d_x, void* stream);

/* Device pointer to the factored LU values (layout per nsg_batch_layout and
 * the topology export: L unscaled, U scaled by the reciprocal pivot, pivots
 * stored as reciprocals — the reference's in-place element values). */
const double* nsg_batch_lu(const nsg_batch* batch);

/* Synchronous copy of all LU values to host memory (lu_offsets[count]
 * doubles). */
int nsg_batch_lu_to_host(const nsg_batch* batch, double* out);

/* ---- Circuits (host) --------------------------------------------------------
 * Typed construction mirroring the reference's Circuit API
 * (src/core/circuit.hpp:179-237) for the devices of the batched DC path:
 * nodes are 0..num_nodes-1 and -1 is ground (Circuit::node("0") == GND).
 * nsg_circuit_finalize mirrors Circuit::finalize (src/core/circuit.cpp:201-283):
 * ngspice load order, branch unknowns after the nodes, sparsity pattern,
 * dead-node placeholders.  Parameters are kept in creation order: resistor
 * {ohms}, capacitor {farads, ic}, DC source {value}, PULSE source {v1, v2,
 * td, tr, tf, pw, per}, PWL source {t0, v0, t1, v1, ...}, diode: the 15
 * values of nsg_diode_param_block (at the circuit temperature).  A diode with RS gets an internal node
 * (posPrime) after the external nodes, in load order, as DIOsetup's
 * CKTmkVolt does; nsg_circuit_info's node count includes it. */
typedef struct nsg_circuit nsg_circuit;

#define NSG_WAVE_DC 0
#define NSG_WAVE_PULSE 1
#define NSG_WAVE_PWL 2

int nsg_circuit_create(int num_nodes, nsg_circuit** out);
void nsg_circuit_free(nsg_circuit* c);
/* Circuit::R (src/core/circuit.hpp:179). */
int nsg_circuit_add_resistor(nsg_circuit* c, int a, int b, double ohms);
/* Circuit::V with a DC value (src/core/circuit.hpp:186). */
int nsg_circuit_add_vsource(nsg_circuit* c, int p, int n, double volts);
/* Circuit::I with a DC value (src/core/circuit.hpp:189). */
int nsg_circuit_add_isource(nsg_circuit* c, int p, int n, double amps);
/* The circuit temperature in kelvin (the reference's options.temp, default
 * 300.15 = TNOM; `.step TEMP` sets it to the step value + 273.15,
 * src/api/neospice.cpp:255-256).  DIOtemp and MOS1temp apply it to every
 * diode and level-1 MOSFET added afterwards, so it must be set before any
 * device is added (NSG_ERR_INVALID otherwise); BSIM4v7 devices are
 * supported at TNOM only. */
int nsg_circuit_set_temperature(nsg_circuit* c, double kelvin);
/* Circuit::D with a level-1 model card D(IS=is N=n) (src/core/circuit.hpp:210;
 * series resistance 0, T = TNOM). */
int nsg_circuit_add_diode(nsg_circuit* c, int anode, int cathode, double is, double n_emission);
/* Circuit::D with the card D(IS N CJO VJ M FC TT) (junction capacitance and
 * transit time; series resistance 0, no sidewall, T = TNOM).  Requires
 * IS > 0, N > 0, CJO >= 0, VJ > 0, 0 <= M < 1, 0 <= FC < 1, TT >= 0.  The
 * reference's defaults (src/devices/dio/dio_setup.cpp:55-82) are CJO 0,
 * VJ 1, M 0.5, FC 0.5, TT 0. */
int nsg_circuit_add_diode_card(nsg_circuit* c, int anode, int cathode, double is,
                               double n_emission, double cjo, double vj, double m, double fc,
                               double tt);
/* The same with reverse breakdown and series resistance: the card D(IS N
 * CJO VJ M FC TT BV IBV NBV RS).  bv NaN means BV not given (no breakdown
 * region); nbv NaN means N (DIOsetup's default); the reference's IBV
 * default is 1e-3; rs 0 means no series resistance.  With BV, requires
 * BV > 0, IBV > 0, NBV > 0; RS >= 0.  The load follows DIOload's breakdown
 * limiting and current (src/devices/dio/dio_load.cpp:158-168, :232-258)
 * and its series-conductance stamps between pos and the internal posPrime
 * (DIOsetup, dio_setup.cpp:232-266). */
int nsg_circuit_add_diode_card_ex(nsg_circuit* c, int anode, int cathode, double is,
                                  double n_emission, double cjo, double vj, double m, double fc,
                                  double tt, double bv, double ibv, double nbv, double rs);
/* The diode parameter block of a card at TNOM (15 doubles into out): IS, N, then
 * DIOtemp's junction capacitance, junction potential, depletion knee FC*VJ,
 * F1, F2, F3, grading coefficient and transit time at T = TNOM
 * (src/devices/dio/dio_temp.cpp:91-292), then 1/0 for BV given, DIOtemp's
 * breakdown voltage matched to IBV (dio_temp.cpp:233-270, the circuit's
 * RELTOL at its default 1e-3), NBV, RS and vt.  bv NaN: no breakdown.  At
 * another circuit temperature IS becomes DIOtemp's saturation current (EG
 * 1.11, XTI 3) and the junction values and vt follow the temperature. */
int nsg_diode_param_block(double is, double n_emission, double cjo, double vj, double m,
                          double fc, double tt, double bv, double ibv, double nbv, double rs,
                          double* out);
/* Circuit::C (src/core/circuit.hpp:180) with an optional IC= value
 * (has_ic != 0). */
int nsg_circuit_add_capacitor(nsg_circuit* c, int a, int b, double farads, int has_ic,
                              double ic);
/* Circuit::V / Circuit::I followed by VSource::set_pulse / set_pwl
 * (src/devices/vsource.hpp, isource.hpp): is_voltage selects V or I, wave is
 * NSG_WAVE_*, values as listed above (PULSE: 7 values, a value <= 0 for tr,
 * tf, pw or per takes the transient's default; PWL: time/value pairs). */
int nsg_circuit_add_source_wave(nsg_circuit* c, int is_voltage, int p, int n, int wave,
                                int nvalues, const double* values);
/* A level-1 MOSFET model card (Circuit::model with ".model NAME NMOS|PMOS
 * (LEVEL=1 ...)", src/core/circuit.hpp:259): type +1 NMOS / -1 PMOS and
 * nparams (key, value) pairs with the MOS1 parameter names of
 * src/devices/mos1/mos1_devsup.cpp:123-159 (vto kp gamma phi lambda rd rs rsh
 * cbd cbs is pb cgso cgdo cgbo cj mj cjsw mjsw js tox ld u0 fc nsub tpg nss
 * tnom; kf, af and level are accepted and ignored).  Nonzero rd / rs (or rsh,
 * one square each) give each MOSFET of the card an internal drain' / source'
 * node after the external nodes, in load order, as MOS1setup does; rd = 0 or
 * rs = 0 given beside a nonzero rsh is rejected.  *model_out receives the
 * model index. */
int nsg_circuit_add_mos1_model(nsg_circuit* c, int type, int nparams, const char* const* keys,
                               const double* values, int* model_out);
/* Circuit::M with W and L (src/core/circuit.hpp:218-219).  Its parameter
 * block has 43 values: W, L, VTO, then the card at the circuit temperature
 * (the MOS1setup / MOS1temp results the device load reads). */
int nsg_circuit_add_mosfet(nsg_circuit* c, int d, int g, int s, int b, int model, double w,
                           double l);
/* A BSIM4v7 (LEVEL=14) model card (Circuit::model with ".model name NMOS
 * (LEVEL=14 ...)", BSIM4v7 model factory src/devices/bsim4v7/
 * bsim4v7_factory.cpp:10-16): type +1 NMOS / -1 PMOS and nparams (key,
 * value) pairs.  Supported: the default card with toxe, vth0 and u0 given
 * (level and version are accepted and ignored); other parameters are
 * rejected (NSG_ERR_INVALID).  *model_out receives the model index. */
int nsg_circuit_add_bsim4_model(nsg_circuit* c, int type, int nparams, const char* const* keys,
                                const double* values, int* model_out);
/* A BSIM4v7 instance (Circuit::M with W and L, src/core/circuit.hpp:218-219,
 * plus the DELVTO instance parameter, src/devices/bsim4v7/
 * bsim4v7_param.cpp:142-144): one finger, no internal nodes.  Its parameter
 * block holds W, L, DELVTO, TOXE, then BSIM4v7setup / BSIM4v7temp's values
 * at the circuit temperature (kernels/bsim4_model.cuh, B4Param). */
int nsg_circuit_add_bsim4(nsg_circuit* c, int d, int g, int s, int b, int model, double w,
                          double l, double delvto);
/* Bulk forms: count devices in one call, arrays of terminals and values,
 * created in array order (identical to count single calls). */
int nsg_circuit_add_capacitors(nsg_circuit* c, int count, const int* a, const int* b,
                               const double* farads);
int nsg_circuit_add_resistors(nsg_circuit* c, int count, const int* a, const int* b,
                              const double* ohms);
int nsg_circuit_add_isources(nsg_circuit* c, int count, const int* p, const int* n,
                             const double* amps);
int nsg_circuit_add_diodes(nsg_circuit* c, int count, const int* anode, const int* cathode,
                           const double* is, const double* n_emission);
int nsg_circuit_finalize(nsg_circuit* c);
int nsg_circuit_info(const nsg_circuit* c, int* num_vars, int* num_nodes, int* nnz,
                     int* num_params);
/* CSC pattern (col_ptr: num_vars+1, row_idx: nnz) and parameters. */
int nsg_circuit_pattern(const nsg_circuit* c, int* col_ptr, int* row_idx);
int nsg_circuit_params(const nsg_circuit* c, double* params);
/* Parameters held so far (finalized or not): the index the next device's
 * first parameter gets. */
int nsg_circuit_param_count(const nsg_circuit* c, int* count);
/* Overwrite one parameter (index into the layout above): a resistance,
 * capacitance, DC source value, a MOSFET's W, L or VTO (block offsets 0-2).
 * Derived entries of a diode or MOSFET block are not recomputed. */
int nsg_circuit_set_param(nsg_circuit* c, int index, double value);
/* The values of a `.step` sweep, as Simulator::run_step_sweep
 * (src/api/neospice.cpp:228-331) produces them: start, start + step, ...
 * (accumulated), while within stop plus a thousandth of |step|.  *count gets
 * the number of values; at most cap are written (cap 0: only the count;
 * NSG_ERR_INVALID when cap is too small or step is 0). */
int nsg_step_values(double start, double stop, double step, int cap, double* values, int* count);
/* Matrix values and rhs of the first DC Newton iteration (MODEDCOP |
 * MODEINITJCT from a zero guess), in slot order -- what the reference's
 * first NeoSolver::numeric orders on. */
int nsg_circuit_initial_matrix(const nsg_circuit* c, double gmin, double* values, double* rhs);
/* Matrix values and rhs of one Newton iteration evaluated on the host, as
 * Circuit::load does it for every device (src/core/newton.cpp:150-170):
 * guess x (num_vars), CKTmode `mode` (ngspice MODE* bits), integrator
 * fields ctx = {ag0, ag1, ag2, xmu_ratio, delta, delta_old1, time}, order
 * and method (0 trapezoidal, 1 Gear); options gmin, reltol, abstol.
 * states: the state ring state0..state2 (3 * nsg_circuit_state_count
 * doubles, updated in place as the loads write state0); mos_rec: 12 values
 * per MOSFET carried from load to load (zero before the first).  For
 * checking device models against the reference on the CPU; circuits with
 * diodes are refused. */
int nsg_circuit_eval_matrix(const nsg_circuit* c, int mode, const double* x, const double* ctx,
                            int order, int method, double gmin, double reltol, double abstol,
                            double* states, double* mos_rec, double* values, double* rhs);
/* Length of one state vector of the circuit (CKTnumStates). */
int nsg_circuit_state_count(const nsg_circuit* c);

/* ---- Batched DC operating point (device) ------------------------------------
 * Simulator::run_dc / solve_dc (src/core/dc.cpp:53-242, newton.cpp:51-419):
 * the direct Newton attempt, then true gmin stepping, gmin stepping, source
 * stepping, gain stepping and pseudo-transient continuation
 * (src/core/convergence.cpp:216-703, 986-1097) for instances it fails on, for `count`
 * circuits in one launch, one thread block per circuit.  symbolic: NSG_SYMBOLIC_PER_INSTANCE orders every circuit on its own
 * first-iteration matrix (bit-identical to the reference's pivots);
 * NSG_SYMBOLIC_PER_PATTERN orders once per distinct sparsity pattern and lets
 * the GPU re-validate the pivots of every instance at its second iteration
 * (a failing instance reports NSG_REORDER).  threads: host threads for the
 * symbolic phase (<= 0: all cores). */
#define NSG_SYMBOLIC_PER_INSTANCE 0
#define NSG_SYMBOLIC_PER_PATTERN 1
typedef struct nsg_dc_batch nsg_dc_batch;

int nsg_dc_batch_create(int count, nsg_circuit* const* circuits, int symbolic, int threads,
                        nsg_dc_batch** out);
void nsg_dc_batch_free(nsg_dc_batch* b);
/* Offsets (count+1 each) of every instance's parameters and solution in the
 * packed arrays nsg_dc_batch_run reads and writes. */
int nsg_dc_batch_layout(const nsg_dc_batch* b, long long* param_offsets,
                        long long* solution_offsets);
/* Totals over instances: unknowns, matrix slots, LU entries, refactor
 * updates; number of distinct symbolic results. */
int nsg_dc_batch_stats(const nsg_dc_batch* b, long long* n, long long* nnz, long long* nnz_lu,
                       long long* updates, int* distinct_topologies);
/* Per-instance sizes (arrays of count): unknowns, matrix slots, LU entries,
 * refactor multiply-subtract updates. */
int nsg_dc_batch_instance_stats(const nsg_dc_batch* b, long long* n, long long* nnz,
                                long long* nnz_lu, long long* updates);
/* SimOptions reltol, vntol, abstol, gmin and itl1 (defaults 1e-3, 1e-6,
 * 1e-12, 1e-12, 100; src/core/types.hpp:24-66). */
int nsg_dc_batch_set_options(nsg_dc_batch* b, double reltol, double vntol, double abstol,
                             double gmin, int max_iter);
/* Which of solve_dc's aids (src/core/dc.cpp:53-242) each instance's
 * operating point runs.  NSG_AID_DIRECT (default): the cascade — the direct
 * attempt, true gmin stepping, gmin stepping, source stepping, gain
 * stepping, pseudo-transient continuation.  NSG_AID_SOURCE / NSG_AID_GAIN /
 * NSG_AID_PSEUDO_TRANSIENT: source_stepping / gain_stepping /
 * pseudo_transient (src/core/convergence.cpp:471-703, 986-1097) alone from
 * the zero guess, as solve_dc runs them after the earlier aids fail (gain
 * stepping scales dependent-source gains, which these circuits do not have,
 * so it ramps a fraction with the sources at full value).  d_iterations
 * then counts that aid's Newton iterations. */
#define NSG_AID_DIRECT 0
#define NSG_AID_SOURCE 1
#define NSG_AID_GAIN 2
#define NSG_AID_PSEUDO_TRANSIENT 3
int nsg_dc_batch_set_first_aid(nsg_dc_batch* b, int aid);
/* Run every instance to convergence.  d_params: packed parameters (device;
 * NULL = the circuits' own values); d_solutions: packed solutions (device),
 * the returned iterate as newton_solve returns it; d_status: 0 converged,
 * 1 no convergence (every aid failed), 102 singular, 103 pivot re-validation
 * failed, 104 a bounded wait gave up; d_iterations: Newton iterations. */
int nsg_dc_batch_run(nsg_dc_batch* b, const double* d_params, double* d_solutions, int* d_status,
                     int* d_iterations, void* stream);
/* Host re-ordering (default on): when an instance's pivots fail the
 * re-validation of a later NeoSolver::numeric, nsg_dc_batch_run waits for the
 * stream, re-orders that instance on the host exactly as the reference's
 * order_and_factor does from the failing step, and resumes it on the device
 * at the same Newton iteration (d_status 103 then no longer appears).  Off:
 * nsg_dc_batch_run stays asynchronous and such instances report 103.
 * nsg_dc_batch_reorders: instances re-ordered so far. */
int nsg_dc_batch_set_reorder(nsg_dc_batch* b, int enable);

/* Replay each run's launch (controller reset + Newton kernel) from a
 * captured CUDA graph: the first run after enabling launches normally, the
 * next captures the launch on an internal stream and later runs with the
 * same d_params / d_solutions / d_status / d_iterations replay it on the
 * caller's stream.  A host re-order (new plans, a grown workspace) drops
 * the graph; it is captured again on a later run.  Results are those of a
 * plain launch, bit for bit. */
int nsg_dc_batch_set_graph(nsg_dc_batch* b, int enable);
/* Update destinations of the dataflow refactor: from the plans' update maps
 * (enable 0, default) or from per-warp row -> position maps in a scratch of
 * count x 16 x max_n int32 (enable != 0), which read L(:, r)'s row indices
 * -- shared by every column that uses r -- instead of one map word per
 * multiply-subtract.  Same values either way.  No counterpart in the
 * reference. */
int nsg_dc_batch_set_row_maps(nsg_dc_batch* b, int enable);
/* Runs that replayed a graph so far. */
int nsg_dc_batch_graph_launches(const nsg_dc_batch* b, long long* count);
int nsg_dc_batch_reorders(const nsg_dc_batch* b, long long* count);
/* After a run (synchronises the device): per instance the method that gave
 * the result, as the reference's ConvergenceMethod (src/core/sim_status.hpp:
 * 0 direct Newton, 1 gmin stepping, 2 source or gain stepping, 3
 * pseudo-transient), and the number of Newton solves it took (either may be
 * NULL). */
int nsg_dc_batch_methods(const nsg_dc_batch* b, int* method, int* solves);

/* Engine (NSG_SOLVER_MARKOWITZ or NSG_SOLVER_AMDLU) of each instance's
 * current plan: make_solver's choice for the circuit (make_solver.cpp:
 * 156-178; NEOSPICE_SOLVER / NEOSPICE_FORCE_AMDLU are read when the batch is
 * created), after any AutoFallbackSolver switch. */
int nsg_dc_batch_engines(const nsg_dc_batch* b, int* engine);

/* DC adjoint: for every instance, the gradient of a scalar loss L with
 * respect to the circuit parameters through the operating point, given
 * d_solutions (the run's solutions) and d_cotangent = dL/dx (packed like the
 * solutions).  The Jacobian is re-evaluated at the solution, factored with
 * the instance's pivots and solved transposed (SparseMatrix::solve_transposed,
 * src/solver/solve.cpp:102-141); then dL/dp = -lambda^T dF/dp for resistances,
 * DC source values and MOSFET W, L and VTO, written to d_grads (packed like
 * the parameters; every other parameter gets 0).  The analytic counterpart of
 * the reference's finite-difference .sens (src/core/sens.cpp:57-140).
 * d_status: 0, or 102 when the Jacobian at the solution is singular. */
int nsg_dc_batch_adjoint(nsg_dc_batch* b, const double* d_params, const double* d_solutions,
                         const double* d_cotangent, double* d_grads, int* d_status, void* stream);

/* ---- Batched transient analysis (device) ------------------------------------
 * solve_transient (src/core/transient.cpp:694-1067) for `count` circuits in one
 * launch, one thread block per circuit, each with its own adaptive timestep:
 * DC operating point (MODETRANOP, with gmin stepping, source stepping and
 * pseudo-transient continuation when the direct attempt fails), then the
 * accept/reject loop of TimeStepController
 * (src/core/timestep.cpp) with trapezoidal / Gear / backward-Euler charge
 * integration and the truncation-error estimate of every charge state.  The
 * DC solver and the transient solver are ordered separately on their own
 * first matrices, as the reference creates two solvers.  Circuits may hold
 * R, C, DC/PULSE/PWL V and I sources, level-1 diodes (with junction
 * capacitance and transit time) and level-1 MOSFETs.  Every accepted timepoint (and
 * t = 0) is written for the `nprobe` unknowns in probes[], at most max_points
 * per circuit. */
typedef struct nsg_tran_batch nsg_tran_batch;

int nsg_tran_batch_create(int count, nsg_circuit* const* circuits, double tstep, double tstop,
                          int max_points, int nprobe, const int* probes, int threads,
                          nsg_tran_batch** out);
void nsg_tran_batch_free(nsg_tran_batch* b);
/* Launch shape of the transient kernel: threads per CTA (128, 256 or 512)
 * and CTAs per SM (128: 8; 256: 4; 512: 2; 0 = that default), or 0, 0 for
 * the automatic choice (512 for a few hundred instances or any instance
 * above 128 unknowns; else 128 or 256, enough for one pass of the device
 * loads).  Tuning only: the shapes give the same results.  No counterpart
 * in the reference. */
int nsg_tran_batch_set_shape(nsg_tran_batch* b, int threads, int blocks_per_sm);
/* Run the whole batch on a stream.  Instances stop for the host when a
 * solver needs ordering -- the transient solver on the first transient
 * iteration's matrix as the device computes it, either solver after a failed
 * pivot re-validation -- so the call waits for the stream, orders those
 * instances as NeoSolver::numeric does and resumes them; it returns when
 * every instance has finished. */
int nsg_tran_batch_run(nsg_tran_batch* b, void* stream);
/* Wait for the device and copy results to host arrays (any may be NULL):
 * times [count*max_points], values [count*max_points*nprobe] (point-major),
 * npoints [count] (points stored: t = 0 and the first accepted timepoints,
 * at most max_points), status [count] (0 ok, 2 DC operating point failed, 3
 * Newton failed at the minimum step, 4 step limit, 104 a bounded wait gave
 * up), stats [count*4] (accepted steps, rejected steps, Newton iterations,
 * DC failure code). */
int nsg_tran_batch_results(const nsg_tran_batch* b, double* times, double* values, int* npoints,
                           int* status, int* stats);
/* Host orderings done so far: the transient solver's first ordering per
 * instance plus every re-ordering after a failed pivot re-validation. */
int nsg_tran_batch_orderings(const nsg_tran_batch* b, long long* count);

/* Engines of each instance's DC and transient solvers (the reference creates
 * one of each, transient.cpp:713, :726), or -1 for a solver not yet ordered. */
int nsg_tran_batch_engines(const nsg_tran_batch* b, int* dc_engine, int* tran_engine);

/* Transient adjoint (no counterpart in the reference, whose sensitivities
 * are DC finite differences, src/core/sens.cpp:57-140, and whose
 * SparseMatrix::solve_transposed, src/solver/solve.cpp:102-141, has no
 * caller).  Recording: with enable != 0 the next nsg_tran_batch_run keeps,
 * per accepted timepoint, the integration formula it used, and the
 * operating point. */
int nsg_tran_batch_record(nsg_tran_batch* b, int enable);
/* Newton tolerances of the adjoint's replay of the recorded steps (the
 * forward run's SimOptions by default; tighter values make the gradient
 * agree with finite differences of the same discrete transient). */
int nsg_tran_batch_set_adjoint_options(nsg_tran_batch* b, double reltol, double vntol,
                                       double abstol, int max_iter);
/* Parameter layout (offsets: count+1) and the parameters the DC preamble
 * and the transient use (host arrays, packed like nsg_circuit_params per
 * instance; any pointer may be NULL). */
int nsg_tran_batch_params(const nsg_tran_batch* b, long long* offsets, double* params_dc,
                          double* params_tran);
/* Gradient of L_i = weight * sum_n (x_n[probe[i]] - target_n)^2 over instance
 * i's recorded timepoints (n = 0 the operating point; d_targets: count *
 * max_points device doubles) with respect to every resistance, capacitance,
 * DC source value and MOSFET W, L, VTO, into d_grads (device, packed like the
 * parameters; 0 elsewhere: waveform-source and diode parameters), d_loss[count]
 * and d_status[count] (0, or a Newton / singular / bounded-wait code).  The
 * replay re-solves the operating point with the replayed parameters, starting
 * from the recorded one.  The steps are replayed with a
 * checkpoint every `every` steps.  d_params_dc / d_params_tran (device, may
 * be NULL: the batch's own) replace the parameters of the replay.  Refused
 * (NSG_ERR_INVALID): no recorded run, a run that filled max_points, or
 * BSIM4v7 devices.  Diode charge and level-1 MOSFET charge (Meyer gate,
 * overlap and bulk-junction capacitance) are in the recursion; diode
 * parameters are not differentiated. */
int nsg_tran_batch_adjoint(nsg_tran_batch* b, const int* probe, const double* d_targets,
                           double weight, int every, const double* d_params_dc,
                           const double* d_params_tran, double* d_grads, double* d_loss,
                           int* d_status, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* NSGPU_H */
