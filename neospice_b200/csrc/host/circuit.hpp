// Host-side circuit topology for the batched Newton loop.
//
// A Circuit is built through typed calls that mirror the reference's Circuit
// API (src/core/circuit.hpp:179-237) for the devices on the GPU path, then
// finalized the way Circuit::finalize does it (src/core/circuit.cpp:201-283):
// ngspice load order, branch indices, sparsity pattern, dead-node
// placeholders.  Finalization also compiles a stamp program: for every matrix
// slot and right-hand-side row, the list of device terms in the order the
// reference's devices add them, so the GPU sums every entry in the same
// sequence of IEEE additions.
#pragma once
#include <cmath>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace nsg {

struct Mos1Integ;  // integrator fields of a device load (kernels/mos1_model.cuh)

// ngspice load rank of each device family (src/core/circuit.cpp:34-59).
enum class DevKind : int32_t {
    Mosfet = 3, Capacitor = 17, Diode = 22, ISource = 31, Resistor = 41, VSource = 50,
    Bsim4 = 1003,  // a MOSFET too: load rank 3 (kind_rank)
};
// The load rank of a device family ("M" devices of every level share 3).
inline int32_t kind_rank(DevKind k) {
    return k == DevKind::Bsim4 ? 3 : static_cast<int32_t>(k);
}

// Independent-source waveforms (src/devices/vsource.cpp:80-131).
enum class Wave : int32_t { DC = 0, Pulse = 1, Pwl = 2 };

// How a constant term value is made from the instance's parameters.
enum TermOp : int32_t {
    kTermRecip = 0,     // +1/p           (resistor conductance)
    kTermNegRecip = 1,  // -(1/p)
    kTermValue = 2,     // +p             (DC source value)
    kTermNegValue = 3,  // -p
    kTermOne = 4,       // +1.0
    kTermMinusOne = 5,  // -1.0
    kTermZero = 6,      // +0.0
    kTermMinusZero = 7, // -0.0
    kTermGmin = 8,      // the dead-node pin conductance (SimOptions::gmin)
};

// Dynamic terms, recomputed every Newton iteration, follow the constants in
// this order: diodes, capacitors, waveform sources.
// Per diode (DIOload's loads, src/devices/dio/dio_load.cpp:392-406, RS = 0):
enum DiodeTerm : int32_t { kDGd = 0, kDGdPlusGspr = 1, kDNegGd = 2, kDCdeq = 3, kDNegCdeq = 4,
                           kDiodeTerms = 5 };
// Per capacitor (Capacitor::evaluate, src/devices/capacitor.cpp:28-100):
enum CapTerm : int32_t { kCGeq = 0, kCNegGeq = 1, kCNegCeq = 2, kCCeq = 3, kCapTerms = 4 };
// Per waveform source: the value and its negation at the current time.
enum SrcTerm : int32_t { kSVal = 0, kSNegVal = 1, kSrcTerms = 2 };
// Per MOSFET: the Mos1Term values of kernels/mos1_model.cuh (22 matrix
// terms in MOS1load's order, then the gate, bulk, drain and source rhs).
// A BSIM4v7 MOSFET (kernels/bsim4_model.cuh) has the same term and
// persistent-value counts (26, 12) and 29 states (BSIM4v7numStates).
constexpr int32_t kMosTerms = 26;
constexpr int32_t kMosStates = 17;  // MOS1numStates
constexpr int32_t kB4States = 29;   // BSIM4v7numStates
constexpr int32_t kMosRec = 12;     // persistent per-load values
enum MosFamily : int32_t { kFamilyMos1 = 0, kFamilyBsim4 = 1 };

struct DeviceRec {
    DevKind kind;
    int32_t created;   // creation index over all devices
    int32_t a, b;      // terminals (0-based node, -1 = ground); MOSFET: drain, gate
    int32_t c, e;      // MOSFET: source, bulk
    int32_t param;     // first parameter index
    int32_t nparam;    // parameter count
    int32_t branch;    // VSource branch unknown, else -1
    Wave wave;         // sources
    bool has_ic;       // capacitors
    // Internal nodes assigned at finalize: a diode's posPrime (RS != 0), a
    // level-1 MOSFET's dNodePrime (prime) and sNodePrime (prime2).
    int32_t prime = -1, prime2 = -1;
};

// A level-1 MOSFET model card: the type (+1 NMOS, -1 PMOS) and the given
// parameters (ngspice names, MOS1mPTable of
// src/devices/mos1/mos1_devsup.cpp:123-159).
struct Mos1Card {
    int32_t type = 1;
    std::vector<std::pair<std::string, double>> params;
};

// The MOS1 parameter block (kernels/mos1_model.cuh, Mos1Param) of one
// instance of `card` with width W and length L at the nominal temperature:
// MOS1setup's defaults and MOS1temp (src/devices/mos1/mos1_setup.cpp,
// mos1_temp.cpp).  Throws std::invalid_argument on an unknown or
// unsupported parameter (RD = 0 or RS = 0 given beside a nonzero RSH).
std::vector<double> mos1_param_block(const Mos1Card& card, double W, double L,
                                     double temp = 300.15);

// A BSIM4v7 (LEVEL=14) model card: the type and the given parameters
// (ngspice names).  Supported: the default card with TOXE, VTH0, U0.
struct Bsim4Card {
    int32_t type = 1;
    std::vector<std::pair<std::string, double>> params;
};

// The BSIM4v7 parameter block (kernels/bsim4_model.cuh, B4Param) of one
// instance of `card` with width W, length L and threshold shift DELVTO at
// the nominal temperature: BSIM4v7setup's defaults and BSIM4v7temp
// (src/devices/bsim4v7/bsim4v7_setup.cpp, bsim4v7_temp.cpp).  Throws
// std::invalid_argument on an unsupported parameter.
std::vector<double> bsim4_param_block(const Bsim4Card& card, double W, double L, double delvto);

// The diode parameter block (DiodeParam of kernels/diode_model.cuh) of the
// card D(IS N CJO VJ M FC TT [BV IBV NBV] [RS]) at the nominal temperature:
// DIOtemp (src/devices/dio/dio_temp.cpp:91-292).  bv NaN: no breakdown (BV
// not given); nbv NaN: N; rs 0: no series resistance.  Throws
// std::invalid_argument outside IS > 0, N > 0, CJO >= 0, VJ > 0,
// 0 <= M < 1, 0 <= FC < 1, TT >= 0, RS >= 0 and, with BV, BV > 0, IBV > 0,
// NBV > 0.
std::vector<double> diode_param_block(double is, double n, double cjo, double vj, double m,
                                      double fc, double tt, double bv = NAN, double ibv = 1e-3,
                                      double nbv = NAN, double rs = 0.0, double temp = 300.15);

class Circuit {
public:
    explicit Circuit(int32_t num_nodes);

    // Parameters of every device are kept in creation order in params():
    // resistor {ohms}; capacitor {farads, ic}; DC source {value}; PULSE
    // source {v1, v2, td, tr, tf, pw, per}; PWL source {t0, v0, t1, v1, ...};
    // diode: the DiodeParam block of kernels/diode_model.cuh.
    int32_t add_resistor(int32_t a, int32_t b, double ohms);
    int32_t add_capacitor(int32_t a, int32_t b, double farads, bool has_ic, double ic);
    int32_t add_vsource(int32_t p, int32_t n, double volts);
    int32_t add_isource(int32_t p, int32_t n, double amps);
    // Waveform sources: is_voltage selects V or I; values per Wave above.
    int32_t add_source_wave(bool is_voltage, int32_t p, int32_t n, Wave wave,
                            const std::vector<double>& values);
    // Level-1 diode (Circuit::D with a `.model D(IS N CJO VJ M FC TT)` card,
    // src/core/circuit.hpp:210-211): IS > 0, N > 0, CJO >= 0, VJ > 0,
    // 0 <= M < 1, 0 <= FC < 1, TT >= 0; DIOsetup's defaults
    // (src/devices/dio/dio_setup.cpp:55-82) for the junction values.
    int32_t add_diode(int32_t anode, int32_t cathode, double is, double n_emission,
                      double cjo = 0.0, double vj = 1.0, double m = 0.5, double fc = 0.5,
                      double tt = 0.0, double bv = NAN, double ibv = 1e-3, double nbv = NAN,
                      double rs = 0.0);
    // Level-1 MOSFET models and instances (Circuit::model,
    // src/core/circuit.hpp:259, and Circuit::M with W and L, :218-219).
    // Returns the model / device index.
    // The circuit temperature in kelvin (the reference's options.temp;
    // default 300.15 = TNOM), applied by DIOtemp / MOS1temp to every device
    // added afterwards; set it before adding devices.  BSIM4v7 devices are
    // supported at TNOM only.
    void set_temperature(double kelvin);
    double temperature() const { return temp_; }
    int32_t add_mos1_model(const Mos1Card& card);
    int32_t add_mosfet(int32_t d, int32_t g, int32_t s, int32_t b, int32_t model, double W,
                       double L);
    // BSIM4v7 models and instances (the reference's LEVEL=14 `.model` and an
    // M instance with W, L and the DELVTO instance parameter,
    // src/devices/bsim4v7/bsim4v7_param.cpp:142-144).
    int32_t add_bsim4_model(const Bsim4Card& card);
    int32_t add_bsim4(int32_t d, int32_t g, int32_t s, int32_t b, int32_t model, double W,
                      double L, double delvto);

    void finalize();
    bool finalized() const { return finalized_; }
    // Circuit::is_linear (src/core/circuit.hpp:171-175): no nonlinear device
    // (diodes and MOSFETs here).
    bool is_linear() const { return diodes_.empty() && mos_.empty(); }
    // Whether any MOSFET is a BSIM4v7 instance (always charge-storing).
    bool has_bsim4() const;

    // Node unknowns: the external nodes, then (after finalize) the devices'
    // internal nodes, as the reference's Circuit::num_nodes counts them.
    int32_t num_nodes() const { return num_nodes_ + num_internal_; }
    int32_t num_vars() const { return num_vars_; }
    int32_t nnz() const { return static_cast<int32_t>(row_idx_.size()); }
    const std::vector<int32_t>& col_ptr() const { return col_ptr_; }
    const std::vector<int32_t>& row_idx() const { return row_idx_; }
    const std::vector<double>& params() const { return params_; }
    std::vector<double>& params_mut() { return params_; }
    const std::vector<int32_t>& dead_nodes() const { return dead_nodes_; }

    // Devices with per-iteration evaluation, in load order.
    struct DiodeRec { int32_t pos, neg, param, state; };  // state: base of kDiodeStates
    struct CapRec { int32_t pos, neg, param, has_ic, state; };  // state: base of {q, i}
    struct SrcRec { int32_t is_voltage, wave, param, nparam; };
    struct MosRec { int32_t d, g, s, b, param, state, family; };
    const std::vector<DiodeRec>& diodes() const { return diodes_; }
    const std::vector<CapRec>& caps() const { return caps_; }
    const std::vector<SrcRec>& wave_sources() const { return wsrc_; }
    const std::vector<MosRec>& mosfets() const { return mos_; }
    int32_t num_states() const { return num_states_; }

    // Stamp program (valid after finalize).
    int32_t n_const_terms() const { return static_cast<int32_t>(term_op_.size()); }
    int32_t diode_term_base() const { return n_const_terms(); }
    int32_t cap_term_base() const {
        return diode_term_base() + kDiodeTerms * static_cast<int32_t>(diodes_.size());
    }
    int32_t src_term_base() const {
        return cap_term_base() + kCapTerms * static_cast<int32_t>(caps_.size());
    }
    int32_t mos_term_base() const {
        return src_term_base() + kSrcTerms * static_cast<int32_t>(wsrc_.size());
    }
    int32_t n_terms() const { return mos_term_base() + kMosTerms * static_cast<int32_t>(mos_.size()); }
    const std::vector<int32_t>& term_op() const { return term_op_; }
    const std::vector<int32_t>& term_param() const { return term_param_; }
    // Per matrix slot / rhs row: ptr (size+1) and term indices, in add order.
    const std::vector<int32_t>& slot_ptr() const { return slot_ptr_; }
    const std::vector<int32_t>& slot_terms() const { return slot_terms_; }
    const std::vector<int32_t>& rhs_ptr() const { return rhs_ptr_; }     // native devices
    const std::vector<int32_t>& rhs_terms() const { return rhs_terms_; }
    const std::vector<int32_t>& ucb_ptr() const { return ucb_ptr_; }     // UCB-style devices
    const std::vector<int32_t>& ucb_terms() const { return ucb_terms_; }

    // Gradient program of the DC adjoint: one record {kind, param, a, b, aux}
    // per differentiable parameter group (kGrad*), a/b the nodes or branch
    // the residual derivative lands on.
    enum GradKind : int32_t { kGradResistor = 1, kGradVSource = 2, kGradISource = 3,
                              kGradMosfet = 4 };
    const std::vector<int32_t>& grad_program() const { return grad_; }

    // Source breakpoints in (0, tstop] after resolving PULSE defaults with
    // (tstep, tstop) (VSource::resolve_defaults / get_breakpoints,
    // src/devices/vsource.cpp:51-78, 233-264), in device order.
    std::vector<double> resolved_params(double tstep, double tstop) const;
    std::vector<double> source_breakpoints(const std::vector<double>& params, double tstop) const;

    // Host evaluation of the matrix and rhs at the first Newton iteration of
    // a DC operating point (MODEDCOP | MODEINITJCT, zero initial guess), with
    // host libm -- the values the reference's first NeoSolver::numeric sees.
    // (MODETRANOP | MODEINITJCT gives the same values for these devices.)
    void initjct_values(std::vector<double>& a, std::vector<double>& rhs,
                        double gmin) const;

    // Host evaluation of the matrix and rhs of one Newton iteration at the
    // guess x in CKTmode `mode`, with the integrator fields ic at time
    // `time`: the same device loads as the GPU kernels' (R, V, I, waveform
    // sources, capacitors, MOSFETs of both families), with host libm.
    // states: the ring state0..state2 (3 * num_states, updated in place as
    // the loads write state0); mos_rec: kMosRec values per MOSFET (the
    // previous load's von, mode, ... ; updated).  Diodes are not supported.
    void eval_values(int mode, const double* x, const Mos1Integ& ic, double time, double gmin,
                     double reltol, double abstol, double* states, double* mos_rec,
                     std::vector<double>& a, std::vector<double>& rhs) const;

private:
    int32_t num_nodes_;
    int32_t num_internal_ = 0;
    double temp_ = 300.15;  // circuit temperature (kelvin): the options' TEMP
    int32_t num_vars_ = 0;
    bool finalized_ = false;
    std::vector<DeviceRec> devices_;
    std::vector<double> params_;
    std::vector<int32_t> col_ptr_, row_idx_, dead_nodes_;
    std::vector<DiodeRec> diodes_;
    std::vector<CapRec> caps_;
    std::vector<SrcRec> wsrc_;
    std::vector<MosRec> mos_;
    std::vector<Mos1Card> mos_models_;
    std::vector<Bsim4Card> b4_models_;
    int32_t num_states_ = 0;
    std::vector<int32_t> term_op_, term_param_, grad_;
    std::vector<int32_t> slot_ptr_, slot_terms_, rhs_ptr_, rhs_terms_, ucb_ptr_, ucb_terms_;

    void check_node(int32_t v) const;
    int32_t add_device(DevKind kind, int32_t a, int32_t b, const std::vector<double>& p,
                       Wave wave = Wave::DC, bool has_ic = false);
    int32_t offset(int32_t r, int32_t c) const;  // -1 when ground or absent
    void const_term_values(std::vector<double>& tv, double gmin) const;
    void sum_program(const std::vector<double>& tv, std::vector<double>* a,
                     std::vector<double>* rhs) const;
};

// Physical constants as the reference's diode shim defines them
// (src/devices/dio/dio_shim.hpp:23, ucb_compat.hpp), and the nominal
// temperature (src/core/types.hpp:18).
constexpr double kKoverQ = 1.38064852e-23 / 1.6021766208e-19;
constexpr double kRoot2 = 1.4142135623730950488;
constexpr double kEuler = 2.7182818284590452354;
constexpr double kTNominal = 300.15;

}  // namespace nsg
