// Load of the level-1 junction diode (no knee currents, no sidewall; at the
// circuit temperature; series resistance RS through an internal node, reverse
// breakdown when BV is given), shared by the host (first-iteration
// values for the symbolic phase) and the GPU Newton kernels: the DC current
// and conductance, and the depletion and diffusion charge of the transient.
// Follows DIOload (src/devices/dio/dio_load.cpp:98-383) and DEVpnjlim
// (src/devices/dio/dio_shim.cpp:101-121) operation for operation, with the
// platform's exp/log.
#pragma once
#include <cmath>

#ifdef __CUDACC__
#define NSG_HD __host__ __device__
#else
#define NSG_HD
#endif

namespace nsg {

// Per-instance diode parameter block: the saturation current, the emission
// coefficient, then DIOtemp's temperature-adjusted capacitance values
// (src/devices/dio/dio_temp.cpp:108-292) at T = TNOM.
enum DiodeParam : int {
    kDpCsat = 0,    // DIOtSatCur (IS * area)
    kDpN = 1,       // N
    kDpCj = 2,      // DIOtJctCap
    kDpPot = 3,     // DIOtJctPot
    kDpDepCap = 4,  // DIOtDepCap (FC * DIOtJctPot)
    kDpF1 = 5,      // DIOtF1
    kDpF2 = 6,      // DIOtF2
    kDpF3 = 7,      // DIOtF3
    kDpGrad = 8,    // DIOtGradingCoeff
    kDpTt = 9,      // DIOtTransitTime
    kDpBrk = 10,    // 1 when BV is given (DIObreakdownVoltageGiven), else 0
    kDpTbv = 11,    // DIOtBrkdwnV (DIOtemp's breakdown voltage matched to IBV)
    kDpNbv = 12,    // NBV (DIObrkdEmissionCoeff; N when not given)
    kDpRs = 13,     // RS (0: no series resistance, posPrime == pos)
    kDpVt = 14,     // vt = CONSTKoverQ * DIOtemp (the device temperature)
    kDiodeParams = 15
};

// Series conductance gspr = DIOtConductance * area of DIOtemp at T = TNOM
// (1 / RS, divided by the unit temperature factor; 0 without RS).
NSG_HD inline double diode_gspr(const double* p) {
    return p[kDpRs] != 0.0 ? (1 / p[kDpRs]) / 1.0 * 1.0 : 0.0;
}

// Reverse breakdown of one diode: whether BV is given, DIOtBrkdwnV and
// vtebrk = NBV * vt.
struct DiodeBrk {
    bool on;
    double tbv, vtebrk;
};

NSG_HD inline DiodeBrk diode_brk(const double* p, double vt) {
    return DiodeBrk{p[kDpBrk] != 0.0, p[kDpTbv], p[kDpNbv] * vt};
}

// Diode state slots (src/devices/dio/dio_def.hpp:160-164).
enum DiodeState : int {
    kDsV = 0,   // DIOvoltage
    kDsI = 1,   // DIOcurrent
    kDsG = 2,   // DIOconduct
    kDsQ = 3,   // DIOcapCharge
    kDsCq = 4,  // DIOcapCurrent
    kDiodeStates = 5
};

NSG_HD inline double pnjlim(double vnew, double vold, double vt, double vcrit, int* icheck) {
    if ((vnew > vcrit) && (fabs(vnew - vold) > (vt + vt))) {
        if (vold > 0) {
            const double arg = (vnew - vold) / vt;
            if (arg > 0) vnew = vold + vt * (2 + log(arg - 2));
            else vnew = vold - vt * (2 + log(2 - arg));
        } else {
            vnew = vt * log(vnew / vt);
        }
        *icheck = 1;
    } else {
        if (vnew < 0) {
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
    }
    return vnew;
}

struct DiodeDC {
    double vd, cd, gd;
    double cdb, gdb;  // bottom-junction current and conductance before gmin
    int check;  // 1: limited / junction-init iteration (counts as non-converged)
};

// Current and conductance at the junction voltage vd, limited against
// vd_old by DEVpnjlim when `limit` (every mode but the junction
// initialisation and MODEINITTRAN; in the breakdown region the limiting
// acts on -(vd + tBrkdwnV) with vtebrk, dio_load.cpp:158-168).  csat =
// area-scaled saturation current at T, vte = N*vt, tvcrit = Vcrit.
NSG_HD inline DiodeDC diode_eval(double vd, bool limit, double vd_old, double csat, double vte,
                                 double tvcrit, double gmin,
                                 const DiodeBrk& bk = DiodeBrk{false, 0.0, 0.0}) {
    DiodeDC r;
    r.check = 1;
    if (limit) {
        const double knee = -bk.tbv + 10 * bk.vtebrk;
        if (bk.on && vd < ((0 < knee) ? 0 : knee)) {  // MIN(0, -tBrkdwnV + 10 vtebrk)
            double vdtemp = -(vd + bk.tbv);
            vdtemp = pnjlim(vdtemp, -(vd_old + bk.tbv), bk.vtebrk, tvcrit, &r.check);
            vd = -(vdtemp + bk.tbv);
        } else {
            vd = pnjlim(vd, vd_old, vte, tvcrit, &r.check);
        }
    }
    double cd, gd;
    if (vd >= -3 * vte) {
        const double evd = exp(vd / vte);
        cd = csat * (evd - 1);
        gd = csat * evd / vte;
    } else if (bk.on && !(vd >= -bk.tbv)) {  // breakdown
        const double evrev = exp(-(bk.tbv + vd) / bk.vtebrk);
        cd = -csat * evrev;
        gd = csat * evrev / bk.vtebrk;
    } else {
        double arg = 3 * vte / (vd * 2.7182818284590452354);
        arg = arg * arg * arg;
        cd = -csat * (1 + arg);
        gd = csat * 3 * arg / vd;
    }
    r.cdb = cd;
    r.gdb = gd;
    cd = cd + 0.0;  // + sidewall current (absent)
    gd = gd + 0.0;
    gd = gd + gmin;
    cd = cd + gmin * vd;
    r.vd = vd;
    r.cd = cd;
    r.gd = gd;
    return r;
}

// The DC operating-point load: Vcrit at MODEINITJCT, else the node voltages
// limited against the previous junction voltage.
NSG_HD inline DiodeDC diode_dc_load(bool initjct, double v_pos, double v_neg, double vd_old,
                                    double csat, double vte, double tvcrit, double gmin,
                                    const DiodeBrk& bk = DiodeBrk{false, 0.0, 0.0}) {
    return diode_eval(initjct ? tvcrit : v_pos - v_neg, !initjct, vd_old, csat, vte, tvcrit, gmin,
                      bk);
}

// Junction charge and capacitance of the charge-storage block of DIOload
// (dio_load.cpp:309-346): depletion charge below / above FC * VJ, plus the
// diffusion charge TT * cdb.  The sidewall terms are zero (no CJSW, no
// sidewall current): their diffusion parts enter as the reference's +0.0
// additions, and adding the zero depletion parts changes no sum.
NSG_HD inline void diode_charge(const double* p, double vd, double cdb, double gdb, double* charge,
                                double* capd) {
    const double czero = p[kDpCj], pot = p[kDpPot], grad = p[kDpGrad], depcap = p[kDpDepCap];
    double qdep, cdep;
    if (vd < depcap) {
        const double arg = 1 - vd / pot;
        const double sarg = exp(-grad * log(arg));
        qdep = pot * czero * (1 - arg * sarg) / (1 - grad);
        cdep = czero * sarg;
    } else {
        const double czof2 = czero / p[kDpF2];
        qdep = czero * p[kDpF1] +
               czof2 * (p[kDpF3] * (vd - depcap) + (grad / (pot + pot)) * (vd * vd - depcap * depcap));
        cdep = czof2 * (p[kDpF3] + grad * vd / pot);
    }
    const double tt = p[kDpTt];
    *charge = tt * cdb + tt * 0.0 + qdep;
    *capd = tt * gdb + tt * 0.0 + cdep;
}

// Vcrit of DIOtemp (src/devices/dio/dio_temp.cpp:209-212).
NSG_HD inline double diode_vcrit(double vte, double csat) {
    return vte * log(vte / (1.4142135623730950488 * csat));
}

}  // namespace nsg
