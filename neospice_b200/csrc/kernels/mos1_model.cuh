// MOS1 (Shichman-Hodges, level 1) device evaluation shared by host and device:
// MOS1load (src/devices/mos1/mos1_load.cpp:21-900) for one instance (the
// node voltages are those of drain' and source', the internal nodes that
// RD / RS / RSH add; the series conductances are stamped between them and
// the terminals), bypass off (the reference's
// MOS1Device::evaluate sets CKTbypass = 0), device gain 1.  The limiting
// helpers follow src/devices/mos1/mos1_shim.cpp:98-204 and the charge
// integration NIintegrate (mos1_shim.cpp:44-73).  Every expression keeps the
// reference's operand order so host and device sums round the same way; the
// transcendental calls (exp, log, sqrt) are the platform's own.
#pragma once
#include <cmath>

#include "diode_model.cuh"  // NSG_HD

namespace nsg {

// Per-device parameter block (in the instance's parameter array): the
// instance geometry and threshold, then the model card at the circuit
// temperature as MOS1setup / MOS1temp leave it (computed by the host).
enum Mos1Param : int {
    kMW = 0, kML, kMVto, kMType, kMM, kMLatDiff, kMLambda, kMGamma, kMPhi, kMTPhi,
    kMEgHalfDiff, kMTTrans, kMTSatCur, kMTSatCurDens, kMDrainArea, kMSourceArea, kMOxCapFactor,
    kMCgso, kMCgdo, kMCgbo, kMSourceVcrit, kMDrainVcrit, kMTBulkPot, kMTDepCap, kMCbd,
    kMCbdsw, kMCbs, kMCbssw, kMF2d, kMF3d, kMF4d, kMF2s, kMF3s, kMF4s, kMMj, kMMjsw, kMVt,
    kMIcVds, kMIcVgs, kMIcVbs, kMOff, kMDrainCond, kMSourceCond,
    kMos1Params
};

// State slots relative to the device's state base (mos1_def.hpp:304-327).
enum Mos1State : int {
    kSVbd = 0, kSVbs = 1, kSVgs = 2, kSVds = 3, kSCapgs = 4, kSQgs = 5, kSCqgs = 6,
    kSCapgd = 7, kSQgd = 8, kSCqgd = 9, kSCapgb = 10, kSQgb = 11, kSCqgb = 12,
    kSQbd = 13, kSCqbd = 14, kSQbs = 15, kSCqbs = 16, kMos1States = 17
};

// Values one load leaves in the instance (MOS1instance fields read by the
// next load's limiting and by the convergence test).
enum Mos1Rec : int {
    kRVon = 0, kRVdsat, kRMode, kRCd, kRCbs, kRCbd, kRGm, kRGds, kRGmbs, kRGbd, kRGbs,
    kRNoncon, kMos1Rec
};

// Matrix terms in MOS1load's add order, then the four rhs terms.
enum Mos1Term : int {
    kTDd = 0, kTGg, kTSs, kTBb, kTDPdp, kTSPsp, kTDdp, kTGb, kTGdp, kTGsp, kTSsp, kTBg, kTBdp,
    kTBsp, kTDPd, kTDPg, kTDPb, kTDPsp, kTSPg, kTSPs, kTSPb, kTSPdp,
    kTRhsG, kTRhsB, kTRhsDP, kTRhsSP, kMos1Terms
};

// CKTmode bits used by the load (ngspice cktdefs.h values).
constexpr int kM1Tran = 0x1, kM1DcOp = 0x10, kM1TranOp = 0x20, kM1DcTranCurve = 0x40,
              kM1InitFloat = 0x100, kM1InitJct = 0x200, kM1InitFix = 0x400,
              kM1InitSmsig = 0x800, kM1InitTran = 0x1000, kM1InitPred = 0x2000,
              kM1Uic = 0x10000;

struct Mos1Integ {      // the integrator fields MOS1load reads
    double ag0, ag1, ag2, xmu_ratio, delta, delta_old1;
    int order, method;
};

// MAX / MIN of ucb_compat.hpp: ((a) > (b) ? (a) : (b)), ((a) < (b) ? (a) : (b)).
NSG_HD inline double m1_max(double a, double b) { return (a > b) ? a : b; }
NSG_HD inline double m1_min(double a, double b) { return (a < b) ? a : b; }

NSG_HD inline double m1_limvds(double vnew, double vold) {
    if (vold >= 3.5) {
        if (vnew > vold) {
            vnew = fmin(vnew, (3 * vold) + 2);
        } else if (vnew < 3.5) {
            vnew = fmax(vnew, 2);
        }
    } else {
        vnew = (vnew > vold) ? fmin(vnew, 4) : fmax(vnew, -.5);
    }
    return vnew;
}

NSG_HD inline double m1_pnjlim(double vnew, double vold, double vt, double vcrit, int* icheck) {
    if ((vnew > vcrit) && (fabs(vnew - vold) > (vt + vt))) {
        if (vold > 0) {
            const double arg = (vnew - vold) / vt;
            vnew = (arg > 0) ? vold + vt * (2 + log(arg - 2)) : vold - vt * (2 + log(2 - arg));
        } else {
            vnew = vt * log(vnew / vt);
        }
        *icheck = 1;
    } else if (vnew < 0) {
        const double arg = (vold > 0) ? -1 * vold - 1 : 2 * vold - 1;
        if (vnew < arg) {
            vnew = arg;
            *icheck = 1;
        } else {
            *icheck = 0;
        }
    } else {
        *icheck = 0;
    }
    return vnew;
}

NSG_HD inline double m1_fetlim(double vnew, double vold, double vto) {
    const double vtsthi = fabs(2 * (vold - vto)) + 2;
    const double vtstlo = fabs(vold - vto) + 1;
    const double vtox = vto + 3.5;
    const double delv = vnew - vold;
    if (vold >= vto) {
        if (vold >= vtox) {
            if (delv <= 0) {
                if (vnew >= vtox) {
                    if (-delv > vtstlo) vnew = vold - vtstlo;
                } else {
                    vnew = fmax(vnew, vto + 2);
                }
            } else if (delv >= vtsthi) {
                vnew = vold + vtsthi;
            }
        } else {
            vnew = (delv <= 0) ? fmax(vnew, vto - .5) : fmin(vnew, vto + 4);
        }
    } else if (delv <= 0) {
        if (-delv > vtsthi) vnew = vold - vtsthi;
    } else {
        const double vtemp = vto + .5;
        if (vnew <= vtemp) {
            if (delv > vtstlo) vnew = vold + vtstlo;
        } else {
            vnew = vtemp;
        }
    }
    return vnew;
}

// Meyer gate capacitances (half of the voltage-dependent part).  T is
// double in the load; the transient adjoint evaluates the same expressions
// on a derivative-carrying number type.
template <class T>
NSG_HD inline void m1_qmeyer(T vgs, T vgd, T von, T vdsat, T* capgs, T* capgd, T* capgb,
                             double phi, double cox) {
    const T vgst = vgs - von;
    vdsat = fmax(vdsat, 0.025);
    if (vgst <= -phi) {
        *capgb = cox / 2;
        *capgs = 0;
        *capgd = 0;
    } else if (vgst <= -phi / 2) {
        *capgb = -vgst * cox / (2 * phi);
        *capgs = 0;
        *capgd = 0;
    } else if (vgst <= 0) {
        *capgb = -vgst * cox / (2 * phi);
        *capgs = vgst * cox / (1.5 * phi) + cox / 3;
        const T vds = vgs - vgd;
        if (vds >= vdsat) {
            *capgd = 0;
        } else {
            const T vddif = 2.0 * vdsat - vds;
            const T vddif1 = vdsat - vds;
            const T vddif2 = vddif * vddif;
            *capgd = *capgs * (1.0 - vdsat * vdsat / vddif2);
            *capgs = *capgs * (1.0 - vddif1 * vddif1 / vddif2);
        }
    } else {
        const T vds = vgs - vgd;
        if (vdsat <= vds) {
            *capgs = cox / 3;
            *capgd = 0;
            *capgb = 0;
        } else {
            const T vddif = 2.0 * vdsat - vds;
            const T vddif1 = vdsat - vds;
            const T vddif2 = vddif * vddif;
            *capgd = cox * (1.0 - vdsat * vdsat / vddif2) / 3;
            *capgs = cox * (1.0 - vddif1 * vddif1 / vddif2) / 3;
            *capgb = 0;
        }
    }
}

// NIintegrate on charge slot q (current at q + 1).
NSG_HD inline void m1_integrate(const Mos1Integ& c, double* s0, const double* s1,
                                const double* s2, int q, double cap, double* geq, double* ceq) {
    const int order = c.order < 1 ? 1 : (c.order > 2 ? 2 : c.order);
    double deriv;
    if (order == 1) {
        deriv = c.ag0 * s0[q] + c.ag1 * s1[q];
    } else if (c.method == 0) {
        deriv = -s1[q + 1] * c.xmu_ratio + c.ag0 * s0[q] + c.ag1 * s1[q];
    } else {
        deriv = c.ag0 * s0[q] + c.ag1 * s1[q] + c.ag2 * s2[q];
    }
    s0[q + 1] = deriv;
    *geq = c.ag0 * cap;
    *ceq = s0[q + 1] - (*geq) * s0[q];
}

// The grading factors of a bulk junction below the depletion limit.  The
// reference tests (mj == mjsw, then mj == .5) for the source side and
// (mj == .5 && mjsw == .5) for the drain side; both give these values.
NSG_HD inline void m1_junction_sargs(double mj, double mjsw, double arg, double* sarg,
                                     double* sargsw) {
    if (mj == .5 && mjsw == .5) {
        *sarg = *sargsw = 1 / sqrt(arg);
        return;
    }
    *sarg = (mj == .5) ? 1 / sqrt(arg) : exp(-mj * log(arg));
    *sargsw = (mjsw == .5) ? 1 / sqrt(arg) : exp(-mjsw * log(arg));
}

// Charge and capacitance of the bulk-drain (drain) or bulk-source junction
// at junction voltage v (MOS1load's depletion charge; zero when the
// junction has no capacitance).
NSG_HD inline void m1_bulk_charge(const double* P, double v, bool drain, double* q, double* cap) {
    const double cz = P[drain ? kMCbd : kMCbs], czsw = P[drain ? kMCbdsw : kMCbssw];
    if (cz == 0 && czsw == 0) {
        *q = 0;
        *cap = 0;
        return;
    }
    if (v < P[kMTDepCap]) {
        const double pb = P[kMTBulkPot], mj = P[kMMj], mjsw = P[kMMjsw];
        const double arg = 1 - v / pb;
        double sarg, sargsw;
        m1_junction_sargs(mj, mjsw, arg, &sarg, &sargsw);
        *q = pb * (cz * (1 - arg * sarg) / (1 - mj) + czsw * (1 - arg * sargsw) / (1 - mjsw));
        *cap = cz * sarg + czsw * sargsw;
    } else if (drain) {
        *q = P[kMF4d] + v * (P[kMF2d] + v * P[kMF3d] / 2);
        *cap = P[kMF2d] + v * P[kMF3d];
    } else {
        *q = P[kMF4s] + v * (P[kMF2s] + v * (P[kMF3s] / 2));
        *cap = P[kMF2s] + P[kMF3s] * v;
    }
}

// One MOS1load of one instance.  P: parameter block; rec: persistent
// instance values; s0/s1/s2: the instance's state slots in the state ring;
// v[4]: node voltages d, g, s, b of the previous iterate (0 for ground);
// t: the kMos1Terms stamp values written in MOS1load's order.
NSG_HD inline void mos1_load(const double* P, double* rec, double* s0, double* s1,
                             const double* s2, int mode, const Mos1Integ& ic, double gmin,
                             const double v[4], double* t) {
    const double type = P[kMType];
    const double vt = P[kMVt];
    const double m = P[kMM];
    const double W = P[kMW];
    int Check = 1;

    const double EffectiveLength = P[kML] - 2 * P[kMLatDiff];
    double DrainSatCur, SourceSatCur;
    if ((P[kMTSatCurDens] == 0) || (P[kMDrainArea] == 0) || (P[kMSourceArea] == 0)) {
        DrainSatCur = m * P[kMTSatCur];
        SourceSatCur = m * P[kMTSatCur];
    } else {
        DrainSatCur = P[kMTSatCurDens] * m * P[kMDrainArea];
        SourceSatCur = P[kMTSatCurDens] * m * P[kMSourceArea];
    }
    const double GateSourceOverlapCap = P[kMCgso] * m * W;
    const double GateDrainOverlapCap = P[kMCgdo] * m * W;
    const double GateBulkOverlapCap = P[kMCgbo] * m * EffectiveLength;
    const double Beta = P[kMTTrans] * m * W / EffectiveLength;
    const double OxideCap = P[kMOxCapFactor] * EffectiveLength * m * W;
    // MOS1temp's tVbi / tVto (mos1_temp.cpp) from the threshold parameter.
    const double tVbi = P[kMVto] - type * (P[kMGamma] * sqrt(P[kMPhi])) + P[kMEgHalfDiff] +
                        type * .5 * (P[kMTPhi] - P[kMPhi]);
    const double tVto = tVbi + type * P[kMGamma] * sqrt(P[kMTPhi]);

    double vbs, vgs, vds, vbd, vgd, vgb;
    double xfact = 0.0;
    const bool off = P[kMOff] != 0.0;
    if ((mode & (kM1InitFloat | kM1InitPred | kM1InitSmsig | kM1InitTran)) ||
        ((mode & kM1InitFix) && !off)) {
        if (mode & (kM1InitPred | kM1InitTran)) {
            xfact = ic.delta / ic.delta_old1;
            s0[kSVbs] = s1[kSVbs];
            vbs = (1 + xfact) * (s1[kSVbs]) - (xfact * (s2[kSVbs]));
            s0[kSVgs] = s1[kSVgs];
            vgs = (1 + xfact) * (s1[kSVgs]) - (xfact * (s2[kSVgs]));
            s0[kSVds] = s1[kSVds];
            vds = (1 + xfact) * (s1[kSVds]) - (xfact * (s2[kSVds]));
            s0[kSVbd] = s0[kSVbs] - s0[kSVds];
        } else {
            vbs = type * (v[3] - v[2]);
            vgs = type * (v[1] - v[2]);
            vds = type * (v[0] - v[2]);
        }
        vbd = vbs - vds;
        vgd = vgs - vds;
        const double vgdo = s0[kSVgs] - s0[kSVds];
        const double von = type * rec[kRVon];
        if (s0[kSVds] >= 0) {
            vgs = m1_fetlim(vgs, s0[kSVgs], von);
            vds = vgs - vgd;
            vds = m1_limvds(vds, s0[kSVds]);
            vgd = vgs - vds;
        } else {
            vgd = m1_fetlim(vgd, vgdo, von);
            vds = vgs - vgd;
            vds = -m1_limvds(-vds, -(s0[kSVds]));
            vgs = vgd + vds;
        }
        if (vds >= 0) {
            vbs = m1_pnjlim(vbs, s0[kSVbs], vt, P[kMSourceVcrit], &Check);
            vbd = vbs - vds;
        } else {
            vbd = m1_pnjlim(vbd, s0[kSVbd], vt, P[kMDrainVcrit], &Check);
            vbs = vbd + vds;
        }
    } else if ((mode & kM1InitJct) && !off) {
        vds = type * P[kMIcVds];
        vgs = type * P[kMIcVgs];
        vbs = type * P[kMIcVbs];
        if ((vds == 0) && (vgs == 0) && (vbs == 0) &&
            ((mode & (kM1Tran | kM1DcOp | kM1DcTranCurve)) || (!(mode & kM1Uic)))) {
            vbs = -1;
            vgs = type * tVto;
            vds = 0;
        }
    } else {
        vbs = vgs = vds = 0;
    }
    vbd = vbs - vds;
    vgd = vgs - vds;
    vgb = vgs - vbs;

    // bulk-source and bulk-drain diodes
    double gbs, cbs, gbd, cbd;
    if (vbs <= -3 * vt) {
        gbs = gmin;
        cbs = gbs * vbs - SourceSatCur;
    } else {
        const double evbs = exp(m1_min(709.0, vbs / vt));
        gbs = SourceSatCur * evbs / vt + gmin;
        cbs = SourceSatCur * (evbs - 1) + gmin * vbs;
    }
    if (vbd <= -3 * vt) {
        gbd = gmin;
        cbd = gbd * vbd - DrainSatCur;
    } else {
        const double evbd = exp(m1_min(709.0, vbd / vt));
        gbd = DrainSatCur * evbd / vt + gmin;
        cbd = DrainSatCur * (evbd - 1) + gmin * vbd;
    }
    const int dmode = (vds >= 0) ? 1 : -1;
    const double dm = static_cast<double>(dmode);

    // drain current (Shichman-Hodges)
    double von, vdsat, cdrain, gm, gds, gmbs;
    {
        const double vbx = (dmode == 1 ? vbs : vbd);
        const double tPhi = P[kMTPhi];
        double sarg;
        if (vbx <= 0) {
            sarg = sqrt(tPhi - vbx);
        } else {
            sarg = sqrt(tPhi);
            sarg = sarg - vbx / (sarg + sarg);
            sarg = m1_max(0, sarg);
        }
        von = (tVbi * type) + P[kMGamma] * sarg;
        const double vgst = (dmode == 1 ? vgs : vgd) - von;
        vdsat = m1_max(vgst, 0);
        const double arg = (sarg <= 0) ? 0 : P[kMGamma] / (sarg + sarg);
        if (vgst <= 0) {
            cdrain = 0;
            gm = 0;
            gds = 0;
            gmbs = 0;
        } else {
            const double lambda = P[kMLambda];
            const double betap = Beta * (1 + lambda * (vds * dm));
            if (vgst <= (vds * dm)) {
                cdrain = betap * vgst * vgst * .5;
                gm = betap * vgst;
                gds = lambda * Beta * vgst * vgst * .5;
                gmbs = gm * arg;
            } else {
                cdrain = betap * (vds * dm) * (vgst - .5 * (vds * dm));
                gm = betap * (vds * dm);
                gds = betap * (vgst - (vds * dm)) +
                      lambda * Beta * (vds * dm) * (vgst - .5 * (vds * dm));
                gmbs = gm * arg;
            }
        }
    }
    rec[kRVon] = type * von;
    rec[kRVdsat] = type * vdsat;
    double cd = dm * cdrain - cbd;

    if (mode & (kM1Tran | kM1TranOp | kM1InitSmsig)) {
        double capbs, capbd;
        m1_bulk_charge(P, vbs, false, &s0[kSQbs], &capbs);
        m1_bulk_charge(P, vbd, true, &s0[kSQbd], &capbd);
        if ((mode & kM1Tran) || ((mode & kM1InitTran) && !(mode & kM1Uic))) {
            double geq, ceq;
            m1_integrate(ic, s0, s1, s2, kSQbd, capbd, &geq, &ceq);
            gbd += geq;
            cbd += s0[kSCqbd];
            cd -= s0[kSCqbd];
            m1_integrate(ic, s0, s1, s2, kSQbs, capbs, &geq, &ceq);
            gbs += geq;
            cbs += s0[kSCqbs];
        }
    }
    const bool noncon = (!off || !(mode & (kM1InitFix | kM1InitSmsig))) && (Check == 1);

    s0[kSVbs] = vbs;
    s0[kSVbd] = vbd;
    s0[kSVgs] = vgs;
    s0[kSVds] = vds;

    double capgs = 0.0, capgd = 0.0, capgb = 0.0;
    if (mode & (kM1Tran | kM1TranOp | kM1InitSmsig)) {
        if (dmode > 0) {
            m1_qmeyer(vgs, vgd, von, vdsat, &s0[kSCapgs], &s0[kSCapgd], &s0[kSCapgb],
                      P[kMTPhi], OxideCap);
        } else {
            m1_qmeyer(vgd, vgs, von, vdsat, &s0[kSCapgd], &s0[kSCapgs], &s0[kSCapgb],
                      P[kMTPhi], OxideCap);
        }
        const double vgs1 = s1[kSVgs];
        const double vgd1 = vgs1 - s1[kSVds];
        const double vgb1 = vgs1 - s1[kSVbs];
        if (mode & (kM1TranOp | kM1InitSmsig)) {
            capgs = 2 * s0[kSCapgs] + GateSourceOverlapCap;
            capgd = 2 * s0[kSCapgd] + GateDrainOverlapCap;
            capgb = 2 * s0[kSCapgb] + GateBulkOverlapCap;
        } else {
            capgs = (s0[kSCapgs] + s1[kSCapgs] + GateSourceOverlapCap);
            capgd = (s0[kSCapgd] + s1[kSCapgd] + GateDrainOverlapCap);
            capgb = (s0[kSCapgb] + s1[kSCapgb] + GateBulkOverlapCap);
        }
        if (mode & (kM1InitPred | kM1InitTran)) {
            s0[kSQgs] = (1 + xfact) * s1[kSQgs] - xfact * s2[kSQgs];
            s0[kSQgd] = (1 + xfact) * s1[kSQgd] - xfact * s2[kSQgd];
            s0[kSQgb] = (1 + xfact) * s1[kSQgb] - xfact * s2[kSQgb];
        } else if (mode & kM1Tran) {
            s0[kSQgs] = (vgs - vgs1) * capgs + s1[kSQgs];
            s0[kSQgd] = (vgd - vgd1) * capgd + s1[kSQgd];
            s0[kSQgb] = (vgb - vgb1) * capgb + s1[kSQgb];
        } else {
            s0[kSQgs] = vgs * capgs;
            s0[kSQgd] = vgd * capgd;
            s0[kSQgb] = vgb * capgb;
        }
    }

    double gcgs, ceqgs, gcgd, ceqgd, gcgb, ceqgb;
    if ((mode & kM1InitTran) || (!(mode & kM1Tran))) {
        gcgs = 0;
        ceqgs = 0;
        gcgd = 0;
        ceqgd = 0;
        gcgb = 0;
        ceqgb = 0;
    } else {
        if (capgs == 0) s0[kSCqgs] = 0;
        if (capgd == 0) s0[kSCqgd] = 0;
        if (capgb == 0) s0[kSCqgb] = 0;
        m1_integrate(ic, s0, s1, s2, kSQgs, capgs, &gcgs, &ceqgs);
        m1_integrate(ic, s0, s1, s2, kSQgd, capgd, &gcgd, &ceqgd);
        m1_integrate(ic, s0, s1, s2, kSQgb, capgb, &gcgb, &ceqgb);
        ceqgs = ceqgs - gcgs * vgs + ic.ag0 * s0[kSQgs];
        ceqgd = ceqgd - gcgd * vgd + ic.ag0 * s0[kSQgd];
        ceqgb = ceqgb - gcgb * vgb + ic.ag0 * s0[kSQgb];
    }

    const double ceqbs = type * (cbs - (gbs) * vbs);
    const double ceqbd = type * (cbd - (gbd) * vbd);
    double xnrm, xrev, cdreq;
    if (dmode >= 0) {
        xnrm = 1;
        xrev = 0;
        cdreq = type * (cdrain - gds * vds - gm * vgs - gmbs * vbs);
    } else {
        xnrm = 0;
        xrev = 1;
        cdreq = -(type) * (cdrain - gds * (-vds) - gm * vgd - gmbs * vbd);
    }
    const double dcond = P[kMDrainCond], scond = P[kMSourceCond];
    const double xnr = xnrm - xrev;
    // rhs updates into the UCB array: rhs[g] -= X is recorded as the term -X
    t[kTRhsG] = -(type * (ceqgs + ceqgb + ceqgd));
    t[kTRhsB] = -(ceqbs + ceqbd - type * ceqgb);
    t[kTRhsDP] = (ceqbd - cdreq + type * ceqgd);
    t[kTRhsSP] = cdreq + ceqbs + type * ceqgs;
    t[kTDd] = dcond;
    t[kTGg] = ((gcgd + gcgs + gcgb));
    t[kTSs] = scond;
    t[kTBb] = (gbd + gbs + gcgb);
    t[kTDPdp] = (dcond + gds + gbd + xrev * (gm + gmbs) + gcgd);
    t[kTSPsp] = (scond + gds + gbs + xnrm * (gm + gmbs) + gcgs);
    t[kTDdp] = (-dcond);
    t[kTGb] = -(gcgb);
    t[kTGdp] = -(gcgd);
    t[kTGsp] = -(gcgs);
    t[kTSsp] = (-scond);
    t[kTBg] = -(gcgb);
    t[kTBdp] = -(gbd);
    t[kTBsp] = -(gbs);
    t[kTDPd] = (-dcond);
    t[kTDPg] = (xnr * gm - gcgd);
    t[kTDPb] = (-gbd + xnr * gmbs);
    t[kTDPsp] = (-gds - xnrm * (gm + gmbs));
    t[kTSPg] = (-xnr * gm - gcgs);
    t[kTSPs] = (-scond);
    t[kTSPb] = (-gbs - xnr * gmbs);
    t[kTSPdp] = (-gds - xrev * (gm + gmbs));

    rec[kRMode] = dm;
    rec[kRCd] = cd;
    rec[kRCbs] = cbs;
    rec[kRCbd] = cbd;
    rec[kRGm] = gm;
    rec[kRGds] = gds;
    rec[kRGmbs] = gmbs;
    rec[kRGbd] = gbd;
    rec[kRGbs] = gbs;
    rec[kRNoncon] = noncon ? 1.0 : 0.0;
}

// MOS1Device::device_converged(solution) (mos1_device.cpp:377-423): no
// limiting at the last load and the drain / bulk currents predicted at the
// new solution within tolerance.  v[4]: new node voltages d, g, s, b.
NSG_HD inline bool mos1_converged(const double* P, const double* rec, const double* s0,
                                  const double v[4], double reltol, double abstol) {
    if (rec[kRNoncon] != 0.0) return false;
    const double type = P[kMType];
    const double vbs = type * (v[3] - v[2]);
    const double vgs = type * (v[1] - v[2]);
    const double vds = type * (v[0] - v[2]);
    const double vbd = vbs - vds;
    const double vgd = vgs - vds;
    const double vgdo = s0[kSVgs] - s0[kSVds];
    const double delvbs = vbs - s0[kSVbs];
    const double delvbd = vbd - s0[kSVbd];
    const double delvgs = vgs - s0[kSVgs];
    const double delvds = vds - s0[kSVds];
    const double delvgd = vgd - vgdo;
    const double cdv = rec[kRCd];
    double cdhat;
    if (rec[kRMode] >= 0) {
        cdhat = cdv - rec[kRGbd] * delvbd + rec[kRGmbs] * delvbs + rec[kRGm] * delvgs +
                rec[kRGds] * delvds;
    } else {
        cdhat = cdv - (rec[kRGbd] - rec[kRGmbs]) * delvbd - rec[kRGm] * delvgd +
                rec[kRGds] * delvds;
    }
    const double cb = rec[kRCbs] + rec[kRCbd];
    const double cbhat = cb + rec[kRGbd] * delvbd + rec[kRGbs] * delvbs;
    // std::max(a, b) == (a < b) ? b : a
    double tol = reltol * (fabs(cdhat) < fabs(cdv) ? fabs(cdv) : fabs(cdhat)) + abstol;
    if (fabs(cdhat - cdv) >= tol) return false;
    tol = reltol * (fabs(cbhat) < fabs(cb) ? fabs(cb) : fabs(cbhat)) + abstol;
    return fabs(cbhat - cb) <= tol;
}

}  // namespace nsg
