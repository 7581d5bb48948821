#include "circuit.hpp"

#include "kernels/diode_model.cuh"

#include <algorithm>
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

int32_t Circuit::add_resistor(int32_t a, int32_t b, double ohms) {
    check_node(a);
    check_node(b);
    if (!(ohms != 0.0)) throw std::invalid_argument("Circuit: zero resistance");
    devices_.push_back({DevKind::Resistor, static_cast<int32_t>(devices_.size()), a, b,
                        static_cast<int32_t>(params_.size()), -1});
    params_.push_back(ohms);
    return devices_.back().created;
}

int32_t Circuit::add_vsource(int32_t p, int32_t n, double volts) {
    check_node(p);
    check_node(n);
    devices_.push_back({DevKind::VSource, static_cast<int32_t>(devices_.size()), p, n,
                        static_cast<int32_t>(params_.size()), -1});
    params_.push_back(volts);
    return devices_.back().created;
}

int32_t Circuit::add_isource(int32_t p, int32_t n, double amps) {
    check_node(p);
    check_node(n);
    devices_.push_back({DevKind::ISource, static_cast<int32_t>(devices_.size()), p, n,
                        static_cast<int32_t>(params_.size()), -1});
    params_.push_back(amps);
    return devices_.back().created;
}

int32_t Circuit::add_diode(int32_t anode, int32_t cathode, double is, double n_emission) {
    check_node(anode);
    check_node(cathode);
    if (!(is > 0.0) || !(n_emission > 0.0))
        throw std::invalid_argument("Circuit: diode needs IS > 0 and N > 0");
    devices_.push_back({DevKind::Diode, static_cast<int32_t>(devices_.size()), anode, cathode,
                        static_cast<int32_t>(params_.size()), -1});
    params_.push_back(is);
    params_.push_back(n_emission);
    return devices_.back().created;
}

int32_t Circuit::offset(int32_t r, int32_t c) const {
    if (r < 0 || c < 0) return -1;
    // binary search in column c
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
        if (x.kind != y.kind) return static_cast<int32_t>(x.kind) < static_cast<int32_t>(y.kind);
        return x.created > y.created;
    });

    // Branch unknowns follow all node unknowns, in load order.
    int32_t next = num_nodes_;
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
                stamp(d.a, d.a); stamp(d.a, d.b); stamp(d.b, d.a); stamp(d.b, d.b);
                break;
            case DevKind::VSource:
                stamp(d.a, d.branch); stamp(d.b, d.branch); stamp(d.branch, d.a); stamp(d.branch, d.b);
                break;
            case DevKind::Diode:  // pos == posPrime (RS = 0)
                stamp(d.a, d.a); stamp(d.b, d.a); stamp(d.a, d.a); stamp(d.a, d.b);
                stamp(d.a, d.a); stamp(d.b, d.b); stamp(d.a, d.a);
                break;
            case DevKind::ISource:
                break;
        }
    }
    std::vector<char> touched(num_vars_, 0);
    for (const auto& [c, r] : ent) touched[r] = touched[c] = 1;
    dead_nodes_.clear();
    for (int32_t i = 0; i < num_nodes_; ++i)
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

    // Stamp program: replay each device's evaluate() in load order.
    const int32_t nnz = static_cast<int32_t>(row_idx_.size());
    std::vector<std::vector<int32_t>> slot(nnz), rhs(num_vars_), ucb(num_vars_);
    term_op_.clear();
    term_param_.clear();
    auto konst = [&](int32_t op, int32_t param) {
        term_op_.push_back(op);
        term_param_.push_back(param);
        return static_cast<int32_t>(term_op_.size()) - 1;
    };
    // Dynamic (per-iteration) terms are recorded as -1 - (diode * kDiodeTerms
    // + which) and renumbered after the constants once their count is known.
    auto dyn_term = [](int32_t diode, int32_t which) { return -1 - (diode * kDiodeTerms + which); };
    auto add_slot = [&](int32_t r, int32_t c, int32_t term) {
        const int32_t off = offset(r, c);
        if (off >= 0) slot[off].push_back(term);
    };
    diodes_.clear();
    for (const auto& d : order) {
        switch (d.kind) {
            case DevKind::Diode: {
                const int32_t id = static_cast<int32_t>(diodes_.size());
                diodes_.push_back({d.a, d.b, d.param});
                // rhs (UCB array): neg += cdeq, posPrime -= cdeq
                if (d.b >= 0) ucb[d.b].push_back(dyn_term(id, kDCdeq));
                if (d.a >= 0) ucb[d.a].push_back(dyn_term(id, kDNegCdeq));
                // matrix, in DIOload's order
                const int32_t zero = konst(kTermZero, -1), mzero = konst(kTermMinusZero, -1);
                auto dslot = [&](int32_t r, int32_t c, int32_t which) {
                    const int32_t off = offset(r, c);
                    if (off >= 0) slot[off].push_back(dyn_term(id, which));
                };
                add_slot(d.a, d.a, zero);                 // PosPos += gspr
                dslot(d.b, d.b, kDGd);                    // NegNeg += gd
                dslot(d.a, d.a, kDGdPlusGspr);            // PosPrimePosPrime += gd + gspr
                add_slot(d.a, d.a, mzero);                // PosPosPrime -= gspr
                dslot(d.b, d.a, kDNegGd);                 // NegPosPrime -= gd
                add_slot(d.a, d.a, mzero);                // PosPrimePos -= gspr
                dslot(d.a, d.b, kDNegGd);                 // PosPrimeNeg -= gd
                break;
            }
            case DevKind::ISource:
                if (d.a >= 0) rhs[d.a].push_back(konst(kTermNegValue, d.param));
                if (d.b >= 0) rhs[d.b].push_back(konst(kTermValue, d.param));
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
                rhs[d.branch].push_back(konst(kTermValue, d.param));
                break;
            }
        }
    }
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

void Circuit::initjct_values(std::vector<double>& a, std::vector<double>& rhs, double gmin) const {
    if (!finalized_) throw std::logic_error("Circuit: not finalized");
    std::vector<double> tv(n_terms(), 0.0);
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
    const double vt = kKoverQ * kTNominal;
    for (size_t d = 0; d < diodes_.size(); ++d) {
        const double csat = params_[diodes_[d].param];
        const double vte = params_[diodes_[d].param + 1] * vt;
        const DiodeDC r = diode_dc_load(true, 0.0, 0.0, 0.0, csat, vte, diode_vcrit(vte, csat), gmin);
        double* t = &tv[n_const_terms() + kDiodeTerms * d];
        const double cdeq = r.cd - r.gd * r.vd;
        t[kDGd] = r.gd;
        t[kDGdPlusGspr] = r.gd + 0.0;
        t[kDNegGd] = -r.gd;
        t[kDCdeq] = cdeq;
        t[kDNegCdeq] = -cdeq;
    }
    a.assign(nnz(), 0.0);
    for (int32_t s = 0; s < nnz(); ++s) {
        double v = 0.0;
        for (int32_t k = slot_ptr_[s]; k < slot_ptr_[s + 1]; ++k) v += tv[slot_terms_[k]];
        a[s] = v;
    }
    rhs.assign(num_vars_, 0.0);
    for (int32_t i = 0; i < num_vars_; ++i) {
        double v = 0.0, u = 0.0;
        for (int32_t k = rhs_ptr_[i]; k < rhs_ptr_[i + 1]; ++k) v += tv[rhs_terms_[k]];
        for (int32_t k = ucb_ptr_[i]; k < ucb_ptr_[i + 1]; ++k) u += tv[ucb_terms_[k]];
        rhs[i] = v + u;
    }
}

}  // namespace nsg
