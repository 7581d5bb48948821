#include "circuit.hpp"

#include "kernels/diode_model.cuh"
#include "kernels/bsim4_model.cuh"
#include "kernels/mos1_model.cuh"
#include "kernels/source_wave.cuh"

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <utility>

namespace nsg {

Circuit::Circuit(int32_t num_nodes) : num_nodes_(num_nodes) {
    if (num_nodes <= 0) throw std::invalid_argument("Circuit: need at least one node");
}

void Circuit::check_node(int32_t v) const {
    if (finalized_) throw std::logic_error("Circuit: already finalized");
    if (v < -1 || v >= num_nodes_)
        throw std::out_of_range("Circuit: node " + std::to_string(v) + " out of range");
}

int32_t Circuit::add_device(DevKind kind, int32_t a, int32_t b, const std::vector<double>& p,
                            Wave wave, bool has_ic) {
    check_node(a);
    check_node(b);
    DeviceRec d;
    d.kind = kind;
    d.created = static_cast<int32_t>(devices_.size());
    d.a = a;
    d.b = b;
    d.param = static_cast<int32_t>(params_.size());
    d.nparam = static_cast<int32_t>(p.size());
    d.c = d.e = -1;
    d.branch = -1;
    d.wave = wave;
    d.has_ic = has_ic;
    devices_.push_back(d);
    params_.insert(params_.end(), p.begin(), p.end());
    return d.created;
}

int32_t Circuit::add_resistor(int32_t a, int32_t b, double ohms) {
    if (!(ohms != 0.0)) throw std::invalid_argument("Circuit: zero resistance");
    return add_device(DevKind::Resistor, a, b, {ohms});
}

int32_t Circuit::add_capacitor(int32_t a, int32_t b, double farads, bool has_ic, double ic) {
    return add_device(DevKind::Capacitor, a, b, {farads, has_ic ? ic : 0.0}, Wave::DC, has_ic);
}

int32_t Circuit::add_vsource(int32_t p, int32_t n, double volts) {
    return add_device(DevKind::VSource, p, n, {volts});
}

int32_t Circuit::add_isource(int32_t p, int32_t n, double amps) {
    return add_device(DevKind::ISource, p, n, {amps});
}

int32_t Circuit::add_source_wave(bool is_voltage, int32_t p, int32_t n, Wave wave,
                                 const std::vector<double>& values) {
    if (wave == Wave::Pulse && values.size() != 7)
        throw std::invalid_argument("Circuit: PULSE takes v1 v2 td tr tf pw per");
    if (wave == Wave::Pwl && (values.size() < 2 || values.size() % 2))
        throw std::invalid_argument("Circuit: PWL takes (time, value) pairs");
    if (wave == Wave::DC && values.size() != 1)
        throw std::invalid_argument("Circuit: DC source takes one value");
    return add_device(is_voltage ? DevKind::VSource : DevKind::ISource, p, n, values, wave);
}

// DIOtemp for one instance of area 1 at T = TNOM = CKTtemp: the grading
// coefficient, the junction potential and capacitance after the (here
// neutral) temperature adjustment, F1..F3 and the depletion-capacitance
// knee, each by the reference's expression.
std::vector<double> diode_param_block(double is, double n, double cjo, double vj, double m,
                                      double fc, double tt, double bv, double ibv, double nbv,
                                      double rs, double temp) {
    if (!(is > 0.0) || !(n > 0.0))
        throw std::invalid_argument("Circuit: diode needs IS > 0 and N > 0");
    if (!(cjo >= 0.0) || !(vj > 0.0) || !(m >= 0.0 && m < 1.0) || !(fc >= 0.0 && fc < 1.0) ||
        !(tt >= 0.0) || !std::isfinite(cjo) || !std::isfinite(vj) || !std::isfinite(tt))
        throw std::invalid_argument(
            "Circuit: diode needs CJO >= 0, VJ > 0, 0 <= M < 1, 0 <= FC < 1, TT >= 0");
    const bool brk = !std::isnan(bv);
    if (std::isnan(nbv)) nbv = n;  // DIOsetup: NBV defaults to N
    if (brk && (!(bv > 0.0) || !std::isfinite(bv) || !(ibv > 0.0) || !std::isfinite(ibv) ||
                !(nbv > 0.0) || !std::isfinite(nbv)))
        throw std::invalid_argument("Circuit: diode breakdown needs BV > 0, IBV > 0, NBV > 0");
    if (!(rs >= 0.0) || !std::isfinite(rs))
        throw std::invalid_argument("Circuit: diode needs RS >= 0");
    constexpr double kBoltz = 1.38064852e-23, kCharge = 1.6021766208e-19, kRefTemp = 300.15;
    if (!(temp > 0.0) || !std::isfinite(temp))
        throw std::invalid_argument("Circuit: temperature must be positive (kelvin)");
    const double tnom = kTNominal, dt = temp - tnom;
    const double vtnom = kKoverQ * tnom;
    const double xfc = std::log(1 - fc);
    double grad = m * (1.0 + (0.0 * dt) + (0.0 * dt * dt));
    if (grad > .9) grad = .9;
    const double vt = kKoverQ * temp;
    const double fact2 = temp / kRefTemp;
    const double egfet = 1.16 - (7.02e-4 * temp * temp) / (temp + 1108);
    const double arg = -egfet / (2 * kBoltz * temp) + 1.1150877 / (kBoltz * (kRefTemp + kRefTemp));
    const double pbfact = -2 * vt * (1.5 * std::log(fact2) + kCharge * arg);
    const double egfet1 = 1.16 - (7.02e-4 * tnom * tnom) / (tnom + 1108);
    const double arg1 = -egfet1 / (kBoltz * 2 * tnom) + 1.1150877 / (2 * kBoltz * kRefTemp);
    const double fact1 = tnom / kRefTemp;
    const double pbfact1 = -2 * vtnom * (1.5 * std::log(fact1) + kCharge * arg1);
    const double pbo = (vj - pbfact1) / fact1;
    const double gmaold = (vj - pbo) / pbo;
    double cj = cjo / (1 + grad * (400e-6 * (tnom - kRefTemp) - gmaold));
    double pot = pbfact + fact2 * pbo;
    const double gmanew = (pot - pbo) / pbo;
    cj *= 1 + grad * (400e-6 * (temp - kRefTemp) - gmanew);
    const double f1 = pot * (1 - std::exp((1 - grad) * xfc)) / (1 - grad);
    double depcap = fc * pot;
    if (depcap > 1.0) {
        pot = 1.0 / fc;
        depcap = fc * pot;
    }
    const double ttt = tt * (1.0 + (0.0 * dt) + (0.0 * dt * dt));
    const double f2 = std::exp((1 + grad) * xfc);
    const double f3 = 1 - fc * (1 + grad);
    // DIOtemp's saturation current at the device temperature (EG 1.11,
    // XTI 3, area 1): IS itself at TNOM.
    const double eg = 1.11, xti = 3.0;
    const double tsat = is * 1.0 * std::exp(((temp / tnom) - 1) * eg / (n * vt) +
                                            xti / n * std::log(temp / tnom));
    std::vector<double> p(kDiodeParams);
    p[kDpCsat] = tsat;
    p[kDpN] = n;
    p[kDpCj] = cj;
    p[kDpPot] = pot;
    p[kDpDepCap] = depcap;
    p[kDpF1] = f1;
    p[kDpF2] = f2;
    p[kDpF3] = f3;
    p[kDpGrad] = grad;
    p[kDpTt] = ttt;
    // DIOtemp's breakdown voltage (dio_temp.cpp:233-270; TLEV = 0, TCV = 0,
    // level 1, the circuit's RELTOL at its default 1e-3): the voltage at
    // which the reverse current matches IBV, by up to 25 fixed-point steps.
    double xbv = 0.0;
    if (brk) {
        const double tbv = bv - 0.0 * dt;
        double cbv = ibv;
        if (cbv < tsat * tbv / vt) {
            cbv = tsat * tbv / vt;
            xbv = tbv;
        } else {
            const double tol = 1e-3 * cbv;
            xbv = tbv - nbv * vt * std::log(1 + cbv / (tsat));
            for (int iter = 0; iter < 25; iter++) {
                xbv = tbv - nbv * vt * std::log(cbv / (tsat) + 1 - xbv / vt);
                const double xcbv = tsat * (std::exp((tbv - xbv) / (nbv * vt)) - 1 + xbv / vt);
                if (std::fabs(xcbv - cbv) <= tol) break;
            }
        }
    }
    p[kDpBrk] = brk ? 1.0 : 0.0;
    p[kDpTbv] = xbv;
    p[kDpNbv] = nbv;
    p[kDpRs] = rs;
    p[kDpVt] = vt;
    return p;
}

int32_t Circuit::add_diode(int32_t anode, int32_t cathode, double is, double n_emission,
                           double cjo, double vj, double m, double fc, double tt, double bv,
                           double ibv, double nbv, double rs) {
    return add_device(DevKind::Diode, anode, cathode,
                      diode_param_block(is, n_emission, cjo, vj, m, fc, tt, bv, ibv, nbv, rs,
                                        temp_));
}

void Circuit::set_temperature(double kelvin) {
    if (finalized_) throw std::logic_error("Circuit: already finalized");
    if (!devices_.empty())
        throw std::logic_error("Circuit: set the temperature before adding devices");
    if (!(kelvin > 0.0) || !std::isfinite(kelvin))
        throw std::invalid_argument("Circuit: temperature must be positive (kelvin)");
    temp_ = kelvin;
}

int32_t Circuit::add_mos1_model(const Mos1Card& card) {
    if (finalized_) throw std::logic_error("Circuit: already finalized");
    (void)mos1_param_block(card, 1e-6, 1e-6);  // validate the card now
    mos_models_.push_back(card);
    return static_cast<int32_t>(mos_models_.size()) - 1;
}

int32_t Circuit::add_mosfet(int32_t d, int32_t g, int32_t s, int32_t b, int32_t model, double W,
                            double L) {
    check_node(s);
    check_node(b);
    if (model < 0 || model >= static_cast<int32_t>(mos_models_.size()))
        throw std::out_of_range("Circuit: unknown MOSFET model " + std::to_string(model));
    if (!(W > 0.0) || !(L > 0.0)) throw std::invalid_argument("Circuit: MOSFET needs W > 0, L > 0");
    const int32_t id =
        add_device(DevKind::Mosfet, d, g, mos1_param_block(mos_models_[model], W, L, temp_));
    devices_.back().c = s;
    devices_.back().e = b;
    return id;
}

int32_t Circuit::add_bsim4_model(const Bsim4Card& card) {
    if (finalized_) throw std::logic_error("Circuit: already finalized");
    (void)bsim4_param_block(card, 1e-6, 1e-7, 0.0);  // validate the card now
    b4_models_.push_back(card);
    return static_cast<int32_t>(b4_models_.size()) - 1;
}

int32_t Circuit::add_bsim4(int32_t d, int32_t g, int32_t s, int32_t b, int32_t model, double W,
                           double L, double delvto) {
    check_node(s);
    check_node(b);
    if (model < 0 || model >= static_cast<int32_t>(b4_models_.size()))
        throw std::out_of_range("Circuit: unknown BSIM4v7 model " + std::to_string(model));
    if (temp_ != kTNominal)
        throw std::invalid_argument("Circuit: BSIM4v7 devices are supported at TNOM only");
    const int32_t id =
        add_device(DevKind::Bsim4, d, g, bsim4_param_block(b4_models_[model], W, L, delvto));
    devices_.back().c = s;
    devices_.back().e = b;
    return id;
}

bool Circuit::has_bsim4() const {
    for (const auto& m : mos_)
        if (m.family == kFamilyBsim4) return true;
    return false;
}

int32_t Circuit::offset(int32_t r, int32_t c) const {
    if (r < 0 || c < 0) return -1;
    const auto b = row_idx_.begin() + col_ptr_[c];
    const auto e = row_idx_.begin() + col_ptr_[c + 1];
    const auto it = std::lower_bound(b, e, r);
    if (it == e || *it != r) throw std::logic_error("Circuit: stamp outside pattern");
    return static_cast<int32_t>(it - row_idx_.begin());
}

void Circuit::finalize() {
    if (finalized_) throw std::logic_error("Circuit: finalize called twice");

    // ngspice load order: by family rank, then newest instance first
    // (Circuit::rebuild_device_load_order, src/core/circuit.cpp:61-103, with
    // the typed API's default model/instance orders).
    std::vector<DeviceRec> order = devices_;
    std::stable_sort(order.begin(), order.end(), [](const DeviceRec& x, const DeviceRec& y) {
        if (kind_rank(x.kind) != kind_rank(y.kind)) return kind_rank(x.kind) < kind_rank(y.kind);
        return x.created > y.created;
    });

    // Internal nodes, in load order after the external nodes (each device's
    // declare_internal_nodes, src/core/circuit.cpp:205-211): a diode with
    // RS gets posPrime (DIOsetup's CKTmkVolt).  Branch unknowns follow all
    // node unknowns, in load order.
    int32_t next = num_nodes_;
    for (auto& d : order) {
        if (d.kind == DevKind::Diode && params_[d.param + kDpRs] != 0.0) d.prime = next++;
        if (d.kind == DevKind::Mosfet) {  // MOS1setup: drain', then source'
            if (params_[d.param + kMDrainCond] != 0.0) d.prime = next++;
            if (params_[d.param + kMSourceCond] != 0.0) d.prime2 = next++;
        }
    }
    num_internal_ = next - num_nodes_;
    for (auto& d : order)
        if (d.kind == DevKind::VSource) d.branch = next++;
    num_vars_ = next;

    // Sparsity pattern: every device's stamp positions, plus a diagonal for
    // nodes that no device touches at all.
    std::vector<std::pair<int32_t, int32_t>> ent;
    auto stamp = [&](int32_t r, int32_t c) {
        if (r >= 0 && c >= 0) ent.emplace_back(c, r);  // (col, row) for sorting
    };
    for (const auto& d : order) {
        switch (d.kind) {
            case DevKind::Resistor:
            case DevKind::Capacitor:
                stamp(d.a, d.a); stamp(d.a, d.b); stamp(d.b, d.a); stamp(d.b, d.b);
                break;
            case DevKind::VSource:
                stamp(d.a, d.branch); stamp(d.b, d.branch); stamp(d.branch, d.a); stamp(d.branch, d.b);
                break;
            case DevKind::Diode:
                if (d.prime < 0) {  // pos == posPrime (RS = 0)
                    stamp(d.a, d.a); stamp(d.b, d.a); stamp(d.a, d.b); stamp(d.b, d.b);
                } else {  // DIOsetup's TSTALLOC list
                    const int32_t P = d.a, N = d.b, Pp = d.prime;
                    stamp(P, Pp); stamp(N, Pp); stamp(Pp, P); stamp(Pp, N);
                    stamp(P, P); stamp(N, N); stamp(Pp, Pp);
                }
                break;
            case DevKind::ISource:
                break;
            case DevKind::Mosfet: {  // MOS1setup's TSTALLOC list
                const int32_t D = d.a, G = d.b, S = d.c, B = d.e;
                const int32_t Dp = d.prime >= 0 ? d.prime : D, Sp = d.prime2 >= 0 ? d.prime2 : S;
                stamp(D, D); stamp(G, G); stamp(S, S); stamp(B, B); stamp(Dp, Dp); stamp(Sp, Sp);
                stamp(D, Dp); stamp(G, B); stamp(G, Dp); stamp(G, Sp); stamp(S, Sp); stamp(B, Dp);
                stamp(B, Sp); stamp(Dp, Sp); stamp(Dp, D); stamp(B, G); stamp(Dp, G); stamp(Sp, G);
                stamp(Sp, S); stamp(Dp, B); stamp(Sp, B); stamp(Sp, Dp);
                break;
            }
            case DevKind::Bsim4: {  // BSIM4v7setup's TSTALLOC list without internal nodes
                const int32_t D = d.a, G = d.b, S = d.c, B = d.e;
                stamp(D, B); stamp(G, B); stamp(S, B); stamp(B, D); stamp(B, G); stamp(B, S);
                stamp(B, B); stamp(D, D); stamp(G, G); stamp(S, S); stamp(D, D); stamp(S, S);
                stamp(D, D); stamp(G, D); stamp(G, S); stamp(S, S); stamp(D, S); stamp(D, D);
                stamp(D, G); stamp(S, G); stamp(S, S); stamp(S, D);
                break;
            }
        }
    }
    std::vector<char> touched(num_vars_, 0);
    for (const auto& [c, r] : ent) touched[r] = touched[c] = 1;
    dead_nodes_.clear();
    for (int32_t i = 0; i < num_nodes(); ++i)
        if (!touched[i]) {
            ent.emplace_back(i, i);
            dead_nodes_.push_back(i);
        }
    std::sort(ent.begin(), ent.end());
    ent.erase(std::unique(ent.begin(), ent.end()), ent.end());
    col_ptr_.assign(num_vars_ + 1, 0);
    row_idx_.clear();
    for (const auto& [c, r] : ent) {
        ++col_ptr_[c + 1];
        row_idx_.push_back(r);
    }
    for (int32_t j = 0; j < num_vars_; ++j) col_ptr_[j + 1] += col_ptr_[j];
    for (int32_t j = 0; j < num_vars_; ++j)
        if (col_ptr_[j + 1] == col_ptr_[j])
            throw std::invalid_argument("Circuit: unknown " + std::to_string(j) +
                                        " has an empty column (floating branch?)");

    // Device tables in load order (state slots assigned in load order, as
    // Circuit::rebind_device_states does).
    diodes_.clear();
    caps_.clear();
    wsrc_.clear();
    mos_.clear();
    std::vector<int32_t> index_in_table(order.size(), -1);
    int32_t state = 0;
    for (size_t k = 0; k < order.size(); ++k) {
        const auto& d = order[k];
        if (d.kind == DevKind::Mosfet || d.kind == DevKind::Bsim4) {
            const bool b4 = d.kind == DevKind::Bsim4;
            index_in_table[k] = static_cast<int32_t>(mos_.size());
            // the load sees drain' and source' (the terminals without RD / RS)
            mos_.push_back({d.prime >= 0 ? d.prime : d.a, d.b, d.prime2 >= 0 ? d.prime2 : d.c, d.e,
                            d.param, state, b4 ? kFamilyBsim4 : kFamilyMos1});
            state += b4 ? kB4States : kMosStates;
        } else if (d.kind == DevKind::Diode) {
            index_in_table[k] = static_cast<int32_t>(diodes_.size());
            diodes_.push_back({d.prime >= 0 ? d.prime : d.a, d.b, d.param, state});
            state += kDiodeStates;
        } else if (d.kind == DevKind::Capacitor) {
            index_in_table[k] = static_cast<int32_t>(caps_.size());
            caps_.push_back({d.a, d.b, d.param, d.has_ic ? 1 : 0, state});
            state += 2;
        } else if ((d.kind == DevKind::VSource || d.kind == DevKind::ISource) && d.wave != Wave::DC) {
            index_in_table[k] = static_cast<int32_t>(wsrc_.size());
            wsrc_.push_back({d.kind == DevKind::VSource ? 1 : 0, static_cast<int32_t>(d.wave),
                             d.param, d.nparam});
        }
    }
    num_states_ = state;

    // Stamp program: replay each device's evaluate() in load order.  Dynamic
    // terms are recorded as -1 - (block offset) and renumbered once the
    // constant count is known.
    const int32_t nnz = static_cast<int32_t>(row_idx_.size());
    std::vector<std::vector<int32_t>> slot(nnz), rhs(num_vars_), ucb(num_vars_);
    term_op_.clear();
    term_param_.clear();
    auto konst = [&](int32_t op, int32_t param) {
        term_op_.push_back(op);
        term_param_.push_back(param);
        return static_cast<int32_t>(term_op_.size()) - 1;
    };
    const int32_t nd = static_cast<int32_t>(diodes_.size());
    const int32_t nc = static_cast<int32_t>(caps_.size());
    auto diode_term = [&](int32_t id, int32_t w) { return -1 - (id * kDiodeTerms + w); };
    auto cap_term = [&](int32_t id, int32_t w) { return -1 - (nd * kDiodeTerms + id * kCapTerms + w); };
    const int32_t nw = static_cast<int32_t>(wsrc_.size());
    auto src_term = [&](int32_t id, int32_t w) {
        return -1 - (nd * kDiodeTerms + nc * kCapTerms + id * kSrcTerms + w);
    };
    auto mos_term = [&](int32_t id, int32_t w) {
        return -1 - (nd * kDiodeTerms + nc * kCapTerms + nw * kSrcTerms + id * kMosTerms + w);
    };
    auto add_slot = [&](int32_t r, int32_t c, int32_t term) {
        const int32_t off = offset(r, c);
        if (off >= 0) slot[off].push_back(term);
    };
    for (size_t k = 0; k < order.size(); ++k) {
        const auto& d = order[k];
        const int32_t id = index_in_table[k];
        switch (d.kind) {
            case DevKind::Mosfet: {
                // MOS1load: the four rhs updates (UCB array: gate, bulk,
                // drain', source'), then the 22 matrix adds in order.
                const int32_t D = d.a, G = d.b, S = d.c, B = d.e;
                const int32_t Dp = d.prime >= 0 ? d.prime : D, Sp = d.prime2 >= 0 ? d.prime2 : S;
                if (G >= 0) ucb[G].push_back(mos_term(id, kTRhsG));
                if (B >= 0) ucb[B].push_back(mos_term(id, kTRhsB));
                if (Dp >= 0) ucb[Dp].push_back(mos_term(id, kTRhsDP));
                if (Sp >= 0) ucb[Sp].push_back(mos_term(id, kTRhsSP));
                const int32_t rc[22][2] = {{D, D},   {G, G},   {S, S},   {B, B},   {Dp, Dp},
                                           {Sp, Sp}, {D, Dp},  {G, B},   {G, Dp},  {G, Sp},
                                           {S, Sp},  {B, G},   {B, Dp},  {B, Sp},  {Dp, D},
                                           {Dp, G},  {Dp, B},  {Dp, Sp}, {Sp, G},  {Sp, S},
                                           {Sp, B},  {Sp, Dp}};
                for (int32_t w = 0; w < 22; ++w) add_slot(rc[w][0], rc[w][1], mos_term(id, w));
                break;
            }
            case DevKind::Bsim4: {
                // BSIM4v7load: the rhs updates (UCB array: dNodePrime,
                // gNodePrime, bNodePrime, sNodePrime), then the 22 matrix
                // adds of the default path in order (B4Term).
                const int32_t D = d.a, G = d.b, S = d.c, B = d.e;
                if (D >= 0) ucb[D].push_back(mos_term(id, kB4TRhsDP));
                if (G >= 0) ucb[G].push_back(mos_term(id, kB4TRhsGP));
                if (B >= 0) ucb[B].push_back(mos_term(id, kB4TRhsBP));
                if (S >= 0) ucb[S].push_back(mos_term(id, kB4TRhsSP));
                const int32_t rc[22][2] = {{G, G}, {G, D}, {G, S}, {G, B}, {D, D}, {D, D},
                                           {D, G}, {D, S}, {D, B}, {D, D}, {D, D}, {S, D},
                                           {S, G}, {S, S}, {S, S}, {S, B}, {S, S}, {S, S},
                                           {B, D}, {B, G}, {B, S}, {B, B}};
                for (int32_t w = 0; w < 22; ++w) add_slot(rc[w][0], rc[w][1], mos_term(id, w));
                break;
            }
            case DevKind::Capacitor:
                add_slot(d.a, d.a, cap_term(id, kCGeq));
                add_slot(d.a, d.b, cap_term(id, kCNegGeq));
                add_slot(d.b, d.a, cap_term(id, kCNegGeq));
                add_slot(d.b, d.b, cap_term(id, kCGeq));
                if (d.a >= 0) rhs[d.a].push_back(cap_term(id, kCNegCeq));
                if (d.b >= 0) rhs[d.b].push_back(cap_term(id, kCCeq));
                break;
            case DevKind::Diode: {
                const int32_t P = d.a, N = d.b, Pp = d.prime >= 0 ? d.prime : d.a;
                // rhs (UCB array): neg += cdeq, posPrime -= cdeq
                if (N >= 0) ucb[N].push_back(diode_term(id, kDCdeq));
                if (Pp >= 0) ucb[Pp].push_back(diode_term(id, kDNegCdeq));
                // matrix, in DIOload's order; gspr = 1 / RS (0.0 without RS)
                int32_t gspr, mgspr;
                if (d.prime >= 0) {
                    gspr = konst(kTermRecip, d.param + kDpRs);
                    mgspr = konst(kTermNegRecip, d.param + kDpRs);
                } else {
                    gspr = konst(kTermZero, -1);
                    mgspr = konst(kTermMinusZero, -1);
                }
                add_slot(P, P, gspr);                              // PosPos += gspr
                add_slot(N, N, diode_term(id, kDGd));              // NegNeg += gd
                add_slot(Pp, Pp, diode_term(id, kDGdPlusGspr));    // PosPrimePosPrime += gd + gspr
                add_slot(P, Pp, mgspr);                            // PosPosPrime -= gspr
                add_slot(N, Pp, diode_term(id, kDNegGd));          // NegPosPrime -= gd
                add_slot(Pp, P, mgspr);                            // PosPrimePos -= gspr
                add_slot(Pp, N, diode_term(id, kDNegGd));          // PosPrimeNeg -= gd
                break;
            }
            case DevKind::ISource:
                if (d.wave == Wave::DC) {
                    if (d.a >= 0) rhs[d.a].push_back(konst(kTermNegValue, d.param));
                    if (d.b >= 0) rhs[d.b].push_back(konst(kTermValue, d.param));
                } else {
                    if (d.a >= 0) rhs[d.a].push_back(src_term(id, kSNegVal));
                    if (d.b >= 0) rhs[d.b].push_back(src_term(id, kSVal));
                }
                break;
            case DevKind::Resistor: {
                const int32_t g = konst(kTermRecip, d.param), mg = konst(kTermNegRecip, d.param);
                add_slot(d.a, d.a, g);
                add_slot(d.a, d.b, mg);
                add_slot(d.b, d.a, mg);
                add_slot(d.b, d.b, g);
                break;
            }
            case DevKind::VSource: {
                const int32_t one = konst(kTermOne, -1), mone = konst(kTermMinusOne, -1);
                add_slot(d.a, d.branch, one);
                add_slot(d.b, d.branch, mone);
                add_slot(d.branch, d.a, one);
                add_slot(d.branch, d.b, mone);
                rhs[d.branch].push_back(d.wave == Wave::DC ? konst(kTermValue, d.param)
                                                           : src_term(id, kSVal));
                break;
            }
        }
    }
    // Gradient program (creation order): resistors, DC sources, MOSFETs.
    grad_.clear();
    for (const auto& d : devices_) {
        if (d.kind == DevKind::Resistor) {
            grad_.insert(grad_.end(), {kGradResistor, d.param, d.a, d.b, 0});
        } else if (d.kind == DevKind::VSource && d.wave == Wave::DC) {
            int32_t br = -1;
            for (const auto& o : order)
                if (o.created == d.created) br = o.branch;
            grad_.insert(grad_.end(), {kGradVSource, d.param, br, -1, 0});
        } else if (d.kind == DevKind::ISource && d.wave == Wave::DC) {
            grad_.insert(grad_.end(), {kGradISource, d.param, d.a, d.b, 0});
        }
    }
    for (size_t m = 0; m < mos_.size(); ++m)
        if (mos_[m].family == kFamilyMos1)
            grad_.insert(grad_.end(), {kGradMosfet, mos_[m].param, mos_[m].d, mos_[m].s,
                                       static_cast<int32_t>(m)});
    const int32_t pin = konst(kTermGmin, -1);
    for (int32_t i : dead_nodes_) slot[offset(i, i)].push_back(pin);

    const int32_t nconst = static_cast<int32_t>(term_op_.size());
    auto flatten = [&](std::vector<std::vector<int32_t>>& lists, std::vector<int32_t>& ptr,
                       std::vector<int32_t>& out) {
        ptr.assign(lists.size() + 1, 0);
        out.clear();
        for (size_t k = 0; k < lists.size(); ++k) {
            for (int32_t t : lists[k]) out.push_back(t >= 0 ? t : nconst + (-1 - t));
            ptr[k + 1] = static_cast<int32_t>(out.size());
        }
    };
    flatten(slot, slot_ptr_, slot_terms_);
    flatten(rhs, rhs_ptr_, rhs_terms_);
    flatten(ucb, ucb_ptr_, ucb_terms_);
    finalized_ = true;
}

std::vector<double> Circuit::resolved_params(double tstep, double tstop) const {
    std::vector<double> out = params_;
    for (const auto& d : devices_) {
        if ((d.kind != DevKind::VSource && d.kind != DevKind::ISource) || d.wave != Wave::Pulse)
            continue;
        double* p = &out[d.param];  // v1 v2 td tr tf pw per
        if (p[3] <= 0) p[3] = tstep;
        if (p[4] <= 0) p[4] = tstep;
        if (p[5] <= 0) p[5] = tstop;
        if (p[6] <= 0) p[6] = tstop;
    }
    return out;
}

std::vector<double> Circuit::source_breakpoints(const std::vector<double>& params,
                                                double tstop) const {
    const double tstart = 0.0;
    std::vector<double> bps;
    for (const auto& d : devices_) {  // the reference walks devices in creation order
        if (d.kind != DevKind::VSource && d.kind != DevKind::ISource) continue;
        const double* p = &params[d.param];
        if (d.wave == Wave::Pwl) {
            for (int32_t k = 0; k + 1 < d.nparam; k += 2)
                if (p[k] > tstart && p[k] <= tstop) bps.push_back(p[k]);
        } else if (d.wave == Wave::Pulse) {
            const double td = p[2], tr = p[3], tf = p[4], pw = p[5], per = p[6];
            if (per <= 0.0) continue;
            const int max_periods = static_cast<int>((tstop - td) / per) + 2;
            for (int k = 0; k < max_periods; ++k) {
                const double t0 = td + k * per;
                if (t0 > tstop) break;
                const double edges[] = {t0, t0 + tr, t0 + tr + pw, t0 + tr + pw + tf};
                for (double e : edges)
                    if (e > tstart && e <= tstop) bps.push_back(e);
            }
        }
    }
    return bps;
}

void Circuit::const_term_values(std::vector<double>& tv, double gmin) const {
    tv.assign(n_terms(), 0.0);
    for (int32_t k = 0; k < n_const_terms(); ++k) {
        const double p = term_param_[k] >= 0 ? params_[term_param_[k]] : 0.0;
        switch (term_op_[k]) {
            case kTermRecip: tv[k] = 1.0 / p; break;
            case kTermNegRecip: tv[k] = -(1.0 / p); break;
            case kTermValue: tv[k] = p; break;
            case kTermNegValue: tv[k] = -p; break;
            case kTermOne: tv[k] = 1.0; break;
            case kTermMinusOne: tv[k] = -1.0; break;
            case kTermZero: tv[k] = 0.0; break;
            case kTermMinusZero: tv[k] = -0.0; break;
            case kTermGmin: tv[k] = gmin; break;
        }
    }
}

void Circuit::sum_program(const std::vector<double>& tv, std::vector<double>* a,
                          std::vector<double>* rhs) const {
    if (a) {
        a->assign(nnz(), 0.0);
        for (int32_t s = 0; s < nnz(); ++s) {
            double v = 0.0;
            for (int32_t k = slot_ptr_[s]; k < slot_ptr_[s + 1]; ++k) v += tv[slot_terms_[k]];
            (*a)[s] = v;
        }
    }
    if (rhs) {
        rhs->assign(num_vars_, 0.0);
        for (int32_t i = 0; i < num_vars_; ++i) {
            double v = 0.0, u = 0.0;
            for (int32_t k = rhs_ptr_[i]; k < rhs_ptr_[i + 1]; ++k) v += tv[rhs_terms_[k]];
            for (int32_t k = ucb_ptr_[i]; k < ucb_ptr_[i + 1]; ++k) u += tv[ucb_terms_[k]];
            (*rhs)[i] = v + u;
        }
    }
}

void Circuit::initjct_values(std::vector<double>& a, std::vector<double>& rhs, double gmin) const {
    if (!finalized_) throw std::logic_error("Circuit: not finalized");
    std::vector<double> tv;
    const_term_values(tv, gmin);
    for (size_t d = 0; d < diodes_.size(); ++d) {
        const double csat = params_[diodes_[d].param];
        const double vt = params_[diodes_[d].param + kDpVt];
        const double vte = params_[diodes_[d].param + 1] * vt;
        const DiodeDC r = diode_dc_load(true, 0.0, 0.0, 0.0, csat, vte, diode_vcrit(vte, csat), gmin,
                                        diode_brk(&params_[diodes_[d].param], vt));
        double* t = &tv[diode_term_base() + kDiodeTerms * d];
        const double cdeq = r.cd - r.gd * r.vd;
        t[kDGd] = r.gd;
        t[kDGdPlusGspr] = r.gd + diode_gspr(&params_[diodes_[d].param]);
        t[kDNegGd] = -r.gd;
        t[kDCdeq] = cdeq;
        t[kDNegCdeq] = -cdeq;
    }
    // MOSFETs at MODEDCOP | MODEINITJCT from zero state.
    {
        std::vector<double> rec(kMosRec, 0.0), st(kB4States, 0.0);
        const Mos1Integ ic{0, 0, 0, 0, 0, 0, 1, 0};
        const double v0[4] = {0, 0, 0, 0};
        for (size_t m = 0; m < mos_.size(); ++m) {
            std::fill(rec.begin(), rec.end(), 0.0);
            std::fill(st.begin(), st.end(), 0.0);
            double* t = &tv[mos_term_base() + kMosTerms * m];
            if (mos_[m].family == kFamilyBsim4)
                bsim4_load(&params_[mos_[m].param], rec.data(), st.data(), st.data(), st.data(),
                           kM1DcOp | kM1InitJct, ic, gmin, 1e-3, 1e-12, v0, t);
            else
                mos1_load(&params_[mos_[m].param], rec.data(), st.data(), st.data(), st.data(),
                          kM1DcOp | kM1InitJct, ic, gmin, v0, t);
        }
    }
    // Waveform sources at t = 0.
    for (size_t s = 0; s < wsrc_.size(); ++s) {
        const double v = wave_value(wsrc_[s].wave, &params_[wsrc_[s].param], wsrc_[s].nparam, 0.0);
        tv[src_term_base() + kSrcTerms * s + kSVal] = v;
        tv[src_term_base() + kSrcTerms * s + kSNegVal] = -v;
    }
    sum_program(tv, &a, &rhs);
}

void Circuit::eval_values(int mode, const double* x, const Mos1Integ& ic, double time,
                          double gmin, double reltol, double abstol, double* states,
                          double* mos_rec, std::vector<double>& a,
                          std::vector<double>& rhs) const {
    if (!finalized_) throw std::logic_error("Circuit: not finalized");
    if (!diodes_.empty()) throw std::invalid_argument("Circuit::eval_values: diodes not supported");
    std::vector<double> tv;
    const_term_values(tv, gmin);
    double* st[3] = {states, states + num_states_, states + 2 * static_cast<size_t>(num_states_)};
    auto volt = [&](int32_t node) { return node >= 0 ? x[node] : 0.0; };
    // Capacitors: the state-vector companion of Capacitor::evaluate
    // (capacitor.cpp:28-100), as the kernels' device loads.
    for (size_t k = 0; k < caps_.size(); ++k) {
        const CapRec& cr = caps_[k];
        const double cap = params_[cr.param];
        double* t = &tv[cap_term_base() + kCapTerms * k];
        const int32_t s = cr.state;
        if (!(mode & (kM1Tran | 0x2 | kM1TranOp))) {
            t[0] = t[1] = t[2] = t[3] = 0.0;
            continue;
        }
        const bool cond1 = ((mode & 0x70) && (mode & kM1InitJct)) ||
                           ((mode & 0x10000) && (mode & kM1InitTran));
        const double vcap = cond1 ? (cr.has_ic ? params_[cr.param + 1] : 0.0)
                                  : volt(cr.pos) - volt(cr.neg);
        if (mode & (kM1Tran | 0x2)) {
            double* s0 = st[0];
            double* s1 = st[1];
            if (mode & kM1InitPred) {
                s0[s] = s1[s];
            } else {
                s0[s] = cap * vcap;
                if (mode & kM1InitTran) s1[s] = s0[s];
            }
            const int order = ic.order < 1 ? 1 : (ic.order > 2 ? 2 : ic.order);
            double deriv;
            if (order == 1) deriv = ic.ag0 * s0[s] + ic.ag1 * s1[s];
            else if (ic.method == 0) deriv = -s1[s + 1] * ic.xmu_ratio + ic.ag0 * s0[s] + ic.ag1 * s1[s];
            else deriv = ic.ag0 * s0[s] + ic.ag1 * s1[s] + ic.ag2 * st[2][s];
            s0[s + 1] = deriv;
            const double geq = ic.ag0 * cap;
            const double ceq = s0[s + 1] - ic.ag0 * s0[s];
            if (mode & kM1InitTran) s1[s + 1] = s0[s + 1];
            t[0] = 1.0 * geq;
            t[1] = -1.0 * geq;
            t[2] = -1.0 * ceq;
            t[3] = 1.0 * ceq;
        } else {
            st[0][s] = cap * vcap;
            t[0] = t[1] = t[2] = t[3] = 0.0;
        }
    }
    for (size_t m = 0; m < mos_.size(); ++m) {
        const MosRec& mr = mos_[m];
        const double vn[4] = {volt(mr.d), volt(mr.g), volt(mr.s), volt(mr.b)};
        double* t = &tv[mos_term_base() + kMosTerms * m];
        double* rec = mos_rec + kMosRec * m;
        if (mr.family == kFamilyBsim4)
            bsim4_load(&params_[mr.param], rec, st[0] + mr.state, st[1] + mr.state,
                       st[2] + mr.state, mode, ic, gmin, reltol, abstol, vn, t);
        else
            mos1_load(&params_[mr.param], rec, st[0] + mr.state, st[1] + mr.state,
                      st[2] + mr.state, mode, ic, gmin, vn, t);
    }
    for (size_t s = 0; s < wsrc_.size(); ++s) {
        const double v = wave_value(wsrc_[s].wave, &params_[wsrc_[s].param], wsrc_[s].nparam, time);
        tv[src_term_base() + kSrcTerms * s + kSVal] = v;
        tv[src_term_base() + kSrcTerms * s + kSNegVal] = -v;
    }
    sum_program(tv, &a, &rhs);
}

}  // namespace nsg
