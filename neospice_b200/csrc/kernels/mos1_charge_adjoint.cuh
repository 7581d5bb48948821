// Derivatives of a level-1 MOSFET's charge model for the transient adjoint.
//
// MOS1load keeps five charges per instance: the Meyer gate charges against
// source, drain and bulk, and the bulk-drain / bulk-source junction
// charges.  The junction charges are functions of one junction voltage
// (m1_bulk_charge gives dq/dv).  The Meyer charges are accumulated,
//   q_n = q_{n-1} + (v_n - v_{n-1}) (h(x_n) + h(x_{n-1}) + overlap)
// (mos1_load.cpp's qgs/qgd/qgb update, the operating point q_0 =
// v_0 (2 h(x_0) + overlap)), with h the half-capacitances m1_qmeyer
// computes from vgs, vds, vbs and the threshold.  The adjoint needs dh/dx
// and dh/dVTO; they come from evaluating the load's own von / vdsat chain
// and m1_qmeyer on Dual4, a forward-mode number carrying four directional
// derivatives (type-scaled vgs, vds, vbs and the card's VTO).
#pragma once
#include <cmath>

#include "mos1_model.cuh"

namespace nsg {

// Dual4 and its arithmetic live in their own namespace: argument-dependent
// lookup finds sqrt / fmax for Dual4 operands (m1_qmeyer's unqualified
// calls), while plain double calls elsewhere in nsg keep the C library's.
namespace ad {

struct Dual4 {
    double v;
    double d[4];
    NSG_HD Dual4(double x = 0.0) : v(x), d{0.0, 0.0, 0.0, 0.0} {}
};

NSG_HD inline Dual4 operator+(const Dual4& a, const Dual4& b) {
    Dual4 r(a.v + b.v);
    for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
NSG_HD inline Dual4 operator-(const Dual4& a, const Dual4& b) {
    Dual4 r(a.v - b.v);
    for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
NSG_HD inline Dual4 operator-(const Dual4& a) {
    Dual4 r(-a.v);
    for (int i = 0; i < 4; ++i) r.d[i] = -a.d[i];
    return r;
}
NSG_HD inline Dual4 operator*(const Dual4& a, const Dual4& b) {
    Dual4 r(a.v * b.v);
    for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
NSG_HD inline Dual4 operator/(const Dual4& a, const Dual4& b) {
    Dual4 r(a.v / b.v);
    for (int i = 0; i < 4; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) / b.v;
    return r;
}
NSG_HD inline bool operator<=(const Dual4& a, const Dual4& b) { return a.v <= b.v; }
NSG_HD inline bool operator>=(const Dual4& a, const Dual4& b) { return a.v >= b.v; }
NSG_HD inline Dual4 sqrt(const Dual4& a) {
    Dual4 r(::sqrt(a.v));
    for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] / (2.0 * r.v);
    return r;
}
NSG_HD inline Dual4 fmax(const Dual4& a, double b) { return (a.v >= b) ? a : Dual4(b); }

}  // namespace ad

using ad::Dual4;

// The Meyer half-capacitances h = (capgs, capgd, capgb) as MOS1load stores
// them at the type-scaled branch voltages vgs, vds, vbs, with d[0..2] their
// derivatives in vgs, vds, vbs and d[3] in the card's VTO (through von).
NSG_HD inline void m1_meyer_dual(const double* P, double vgs0, double vds0, double vbs0,
                                 Dual4 h[3]) {
    const double type = P[kMType];
    Dual4 vgs(vgs0), vds(vds0), vbs(vbs0);
    vgs.d[0] = 1.0;
    vds.d[1] = 1.0;
    vbs.d[2] = 1.0;
    const Dual4 vbd = vbs - vds, vgd = vgs - vds;
    const int dmode = (vds0 >= 0) ? 1 : -1;
    const double EffectiveLength = P[kML] - 2 * P[kMLatDiff];
    const double OxideCap = P[kMOxCapFactor] * EffectiveLength * P[kMM] * P[kMW];
    const double tVbi = P[kMVto] - type * (P[kMGamma] * ::sqrt(P[kMPhi])) + P[kMEgHalfDiff] +
                        type * .5 * (P[kMTPhi] - P[kMPhi]);
    Dual4 vbi(tVbi * type);
    vbi.d[3] = type;  // d(tVbi * type) / dVTO
    const Dual4 vbx = (dmode == 1) ? vbs : vbd;
    const double tPhi = P[kMTPhi];
    Dual4 sarg;
    if (vbx.v <= 0) {
        sarg = sqrt(Dual4(tPhi) - vbx);
    } else {
        const double s = ::sqrt(tPhi);
        sarg = Dual4(s) - vbx / Dual4(s + s);
        if (0 > sarg.v) sarg = Dual4(0.0);
    }
    const Dual4 von = vbi + Dual4(P[kMGamma]) * sarg;
    const Dual4 vgst = ((dmode == 1) ? vgs : vgd) - von;
    const Dual4 vdsat = (vgst.v > 0) ? vgst : Dual4(0.0);
    if (dmode > 0)
        m1_qmeyer(vgs, vgd, von, vdsat, &h[0], &h[1], &h[2], tPhi, OxideCap);
    else
        m1_qmeyer(vgd, vgs, von, vdsat, &h[1], &h[0], &h[2], tPhi, OxideCap);
}

// d h / d(node voltages d, g, s, b) from the branch-voltage derivatives.
NSG_HD inline void m1_node_grad(const Dual4& h, double type, double gn[4]) {
    gn[0] = type * h.d[1];
    gn[1] = type * h.d[0];
    gn[3] = type * h.d[2];
    gn[2] = -(gn[0] + gn[1] + gn[3]);
}

// The stamp term (Mos1Term) at row terminal r, column terminal q (0..3 =
// d, g, s, b); with RD = RS = 0 the primed nodes are the terminals.
NSG_HD inline int m1_term_at(int r, int q) {
    switch (r * 4 + q) {
        case 0: return kTDPdp;
        case 1: return kTDPg;
        case 2: return kTDPsp;
        case 3: return kTDPb;
        case 4: return kTGdp;
        case 5: return kTGg;
        case 6: return kTGsp;
        case 7: return kTGb;
        case 8: return kTSPdp;
        case 9: return kTSPg;
        case 10: return kTSPsp;
        case 11: return kTSPb;
        case 12: return kTBdp;
        case 13: return kTBg;
        case 14: return kTBsp;
        default: return kTBb;
    }
}

// Charge units of one MOSFET, in this order: Meyer gate-source, gate-drain,
// gate-bulk, then the bulk-drain and bulk-source junctions.  Terminals of
// each unit (the charge's positive and negative side) and, for the Meyer
// units, the state slot of the half-capacitance.
NSG_HD inline int m1_unit_pos(int j) { return j < 3 ? 1 : 3; }
NSG_HD inline int m1_unit_neg(int j) {
    switch (j) {
        case 0: return 2;
        case 1: return 0;
        case 2: return 3;
        case 3: return 0;
        default: return 2;
    }
}
NSG_HD inline int m1_unit_cap_slot(int j) {
    return j == 0 ? kSCapgs : (j == 1 ? kSCapgd : kSCapgb);
}
constexpr int kMos1ChargeUnits = 5;

// Overlap capacitance of Meyer unit j and its derivatives in W and L.
NSG_HD inline double m1_overlap(const double* P, int j, double* dW, double* dL) {
    const double leff = P[kML] - 2 * P[kMLatDiff];
    double o;
    if (j == 0) o = P[kMCgso] * P[kMM] * P[kMW];
    else if (j == 1) o = P[kMCgdo] * P[kMM] * P[kMW];
    else o = P[kMCgbo] * P[kMM] * leff;
    *dW = (j < 2) ? o / P[kMW] : 0.0;
    *dL = (j == 2) ? o / leff : 0.0;
    return o;
}

// True when the instance carries any charge (gate oxide, overlap or
// junction capacitance).
NSG_HD inline bool m1_has_charge(const double* P) {
    return P[kMOxCapFactor] != 0 || P[kMCgso] != 0 || P[kMCgdo] != 0 || P[kMCgbo] != 0 ||
           P[kMCbd] != 0 || P[kMCbdsw] != 0 || P[kMCbs] != 0 || P[kMCbssw] != 0;
}

}  // namespace nsg
