// BSIM4.7 (BSIM4v7, LEVEL=14) device evaluation shared by host and device:
// BSIM4v7load (src/devices/bsim4v7/bsim4v7_load.cpp:69-5107) for one
// instance on the path a default model card takes -- capMod 2 (charge
// thickness model), mobMod 0, dioMod 1, rgateMod = rbodyMod = rdsMod = 0
// (no internal nodes), trnqsMod = acnqsMod = 0, igcMod = igbMod = 0,
// gidlMod 0 with AGIDL = AGISL = 0, no substrate current (ALPHA0 = ALPHA1 =
// 0), no source-end velocity limit, no velocity overshoot, no poly depletion
// (NGATE = 0), no pocket-implant or DITS threshold shifts, bypass off (the
// reference's adapter sets CKTbypass = 0), device multiplier 1.  The host
// (host/bsim4_card.cpp) refuses cards that leave this path.  Terms that are
// identically zero on it (gate tunnelling, GIDL/GISL, trap-assisted
// tunnelling, the NQS charge) are left out; every other expression keeps the
// reference's operand order so host and device round alike.  Limiting and
// charge integration are the MOS1 helpers (the same DEVfetlim, DEVlimvds,
// DEVpnjlim and NIintegrate, bsim4v7_shim.cpp).
#pragma once
#include <cmath>

#include "mos1_model.cuh"

namespace nsg {

// Per-device parameter block: the instance inputs, then every model,
// size-dependent and instance value the load reads, as BSIM4v7setup and
// BSIM4v7temp leave them at the circuit temperature (host-computed).
enum B4Param : int {
    kB4W = 0, kB4L, kB4Delvto, kB4Toxe,
    kB4Type, kB4IcVds, kB4IcVgs, kB4IcVbs, kB4Off,
    kB4Vtm, kB4Vtm0, kB4TempRatio, kB4Coxe, kB4Coxp, kB4Toxp, kB4Factor1, kB4Vcrit, kB4Ados,
    kB4Bdos, kB4Xpart,
    kB4Leff, kB4Weff, kB4LeffCV, kB4WeffCV, kB4WeffCJ, kB4Phi, kB4SqrtPhi, kB4Xdep0, kB4Vbi,
    kB4Dvt0, kB4Dvt1, kB4Dvt2, kB4Dvt0w, kB4Dvt1w, kB4Dvt2w, kB4Lpe0, kB4Lpeb, kB4K1, kB4K1ox,
    kB4K3, kB4K3b, kB4Kt1, kB4Kt1l, kB4Kt2, kB4W0, kB4Etab, kB4Theta0vb0, kB4Cit, kB4Nfactor,
    kB4Cdsc, kB4Cdscb, kB4Cdscd, kB4Mstar, kB4Voffcbn, kB4Cdep0, kB4Dwg, kB4Dwb, kB4Prwg,
    kB4Prwb, kB4Rds0, kB4Rdswmin, kB4Xj, kB4A0, kB4Ags, kB4B0, kB4B1, kB4Keta, kB4Ua, kB4Ub,
    kB4Uc, kB4Ud, kB4A1, kB4A2, kB4Delta, kB4Pclm, kB4Litl, kB4ThetaRout, kB4Pdiblb, kB4Pscbe1,
    kB4Pscbe2,
    kB4Vth0, kB4K2ox, kB4Eta0, kB4U0temp, kB4Vsattemp, kB4Vtfbphi2, kB4Vbsc, kB4Vfbzb,
    kB4Voffcv, kB4Noff, kB4Acde, kB4Ldeb, kB4Moin, kB4AbulkCVfactor, kB4Cgdl, kB4Cgsl,
    kB4Ckappad, kB4Ckappas, kB4Cgdo, kB4Cgso, kB4Cgbo,
    kB4SatCurS, kB4SatCurD, kB4NjS, kB4NjD, kB4VjsmFwd, kB4IVjsmFwd, kB4VjdmFwd, kB4IVjdmFwd,
    kB4Czbs, kB4Czbssw, kB4Czbsswg, kB4Czbd, kB4Czbdsw, kB4Czbdswg, kB4PhiBS, kB4PhiBSWS,
    kB4PhiBSWGS, kB4PhiBD, kB4PhiBSWD, kB4PhiBSWGD, kB4MJS, kB4MJSWS, kB4MJSWGS, kB4MJD,
    kB4MJSWD, kB4MJSWGD,
    kBsim4Params
};

// State slots relative to the device's state base (bsim4v7_def.hpp:514-547).
enum B4State : int {
    kB4SVbd = 0, kB4SVbs, kB4SVgs, kB4SVds, kB4SVdbs, kB4SVdbd, kB4SVsbs, kB4SVges, kB4SVgms,
    kB4SVses, kB4SVdes, kB4SQb, kB4SCqb, kB4SQg, kB4SCqg, kB4SQd, kB4SCqd, kB4SQgmid,
    kB4SCqgmid, kB4SQbs, kB4SCqbs, kB4SQbd, kB4SCqbd, kB4SQcheq, kB4SCqcheq, kB4SQcdump,
    kB4SCqcdump, kB4SQdef, kB4SQs, kBsim4States = 29
};

// Values one load leaves in the instance for the next load's convergence
// predictions and limiting.
enum B4Rec : int {
    kB4RVon = 0, kB4RMode, kB4RCd, kB4RCbs, kB4RCbd, kB4RGbs, kB4RGbd, kB4RGm, kB4RGds,
    kB4RGmbs, kB4RVdsat, kB4RNoncon, kBsim4Rec
};

// Matrix terms in BSIM4v7load's add order (rgateMod 0, rdsMod 0, rbodyMod 0),
// then the four rhs terms (dNodePrime, gNodePrime, bNodePrime,
// sNodePrime).  GIDL/GISL adds (identically zero here) are not kept.
enum B4Term : int {
    kB4TGPgp = 0, kB4TGPdp, kB4TGPsp, kB4TGPbp, kB4TDPdp, kB4TDPd, kB4TDPgp, kB4TDPsp, kB4TDPbp,
    kB4TDdp, kB4TDd, kB4TSPdp, kB4TSPgp, kB4TSPsp, kB4TSPs, kB4TSPbp, kB4TSsp, kB4TSs, kB4TBPdp,
    kB4TBPgp, kB4TBPsp, kB4TBPbp,
    kB4TRhsDP, kB4TRhsGP, kB4TRhsBP, kB4TRhsSP, kBsim4Terms
};

// The load's constants (bsim4v7_load.cpp:37-51).
constexpr double kB4MaxExp = 5.834617425e14;
constexpr double kB4MinExp = 1.713908431e-15;
constexpr double kB4ExpThreshold = 34.0;
constexpr double kB4Epssi = 1.03594e-10;
constexpr double kB4ChargeQ = 1.60219e-19;
constexpr double kB4Delta3 = 0.02;
constexpr double kB4Delta4 = 0.02;
constexpr double kB4Delta1 = 0.02;
// CONSTvt0 of ucb_compat.hpp.
constexpr double kB4Vt0 = 1.38064852e-23 * 300.15 / 1.6021766208e-19;

// (1 + e^x... ) helper of the short-channel terms: T1 / (T2^2 + 2 T1 MIN_EXP)
// with T1 = exp(x), T2 = T1 - 1 (x < EXP_THRESHOLD), else 1 / (MAX_EXP - 2).
NSG_HD inline double b4_theta(double x, double* dfac) {
    if (x < kB4ExpThreshold) {
        const double T1 = exp(x);
        const double T2 = T1 - 1.0;
        const double T3 = T2 * T2;
        const double T4 = T3 + 2.0 * T1 * kB4MinExp;
        if (dfac) *dfac = T1 * (T4 - 2.0 * T1 * (T2 + kB4MinExp)) / T4 / T4;
        return T1 / T4;
    }
    if (dfac) *dfac = 0.0;
    return 1.0 / (kB4MaxExp - 2.0);
}

// Depletion charge and capacitance of one junction bottom / sidewall /
// gate-sidewall triple at reverse bias (the vbx < 0 branch).
NSG_HD inline void b4_junction_reverse(double v, double cz, double czsw, double czswg,
                                       double phi, double phisw, double phiswg, double mj,
                                       double mjsw, double mjswg, double* q, double* cap) {
    if (cz > 0.0) {
        const double arg = 1.0 - v / phi;
        const double sarg = (mj == 0.5) ? 1.0 / sqrt(arg) : exp(-mj * log(arg));
        *q = phi * cz * (1.0 - arg * sarg) / (1.0 - mj);
        *cap = cz * sarg;
    } else {
        *q = 0.0;
        *cap = 0.0;
    }
    if (czsw > 0.0) {
        const double arg = 1.0 - v / phisw;
        const double sarg = (mjsw == 0.5) ? 1.0 / sqrt(arg) : exp(-mjsw * log(arg));
        *q += phisw * czsw * (1.0 - arg * sarg) / (1.0 - mjsw);
        *cap += czsw * sarg;
    }
    if (czswg > 0.0) {
        const double arg = 1.0 - v / phiswg;
        const double sarg = (mjswg == 0.5) ? 1.0 / sqrt(arg) : exp(-mjswg * log(arg));
        *q += phiswg * czswg * (1.0 - arg * sarg) / (1.0 - mjswg);
        *cap += czswg * sarg;
    }
}

// Junction diode current (dioMod 1) of one side.
NSG_HD inline void b4_junction_current(double v, double isat, double nvtm, double vjmf,
                                       double ivjmf, double gmin, double* g, double* c) {
    if (isat <= 0.0) {
        *g = gmin;
        *c = *g * v;
        return;
    }
    const double T2 = v / nvtm;
    if (T2 < -kB4ExpThreshold) {
        *g = gmin;
        *c = isat * (kB4MinExp - 1.0) + gmin * v;
    } else if (v <= vjmf) {
        const double ev = exp(T2);
        *g = isat * ev / nvtm + gmin;
        *c = isat * (ev - 1.0) + gmin * v;
    } else {
        const double T0 = ivjmf / nvtm;
        *g = T0 + gmin;
        *c = ivjmf - isat + T0 * (v - vjmf) + gmin * v;
    }
}

// Overlap charge and capacitance of one side (capMod 1 and 2).
NSG_HD inline void b4_overlap(double vx, double cgxo, double weffcv, double cgxl, double ckappa,
                              double* c, double* q) {
    const double T0 = vx + kB4Delta1;
    const double T1 = sqrt(T0 * T0 + 4.0 * kB4Delta1);
    const double T2 = 0.5 * (T0 - T1);
    const double T3 = weffcv * cgxl;
    const double T4 = sqrt(1.0 - 4.0 * T2 / ckappa);
    *c = cgxo + T3 - T3 * (1.0 - 1.0 / T4) * (0.5 - 0.5 * T0 / T1);
    *q = (cgxo + T3) * vx - T3 * (T2 + 0.5 * ckappa * (T4 - 1.0));
}

// One BSIM4v7load of one instance.  P: parameter block; rec: persistent
// instance values; s0/s1/s2: the instance's state slots; v[4]: node
// voltages d, g, s, b of the previous iterate (0 for ground); reltol /
// abstol: the convergence test's tolerances; t: the kBsim4Terms stamp
// values.  rec[kB4RNoncon] receives 1 when the instance is not converged.
NSG_HD inline void bsim4_load(const double* P, double* rec, double* s0, double* s1,
                              const double* s2, int mode, const Mos1Integ& ic, double gmin,
                              double reltol, double abstol, const double v[4], double* t) {
    const double type = P[kB4Type];
    const bool off = P[kB4Off] != 0.0;
    const bool charge =
        (mode & (kM1DcTranCurve | kM1Tran | kM1InitSmsig)) || ((mode & kM1TranOp) && (mode & kM1Uic));
    int Check = 1;

    // --- terminal voltages (bsim4v7_load.cpp:237-484) ---
    double vds, vgs, vbs, vges, vgms, vdbs, vsbs, vses, vdes;
    double cdhat = 0.0, cbhat = 0.0, Idtot = 0.0, Ibtot = 0.0;
    bool predicted = false;
    if (mode & kM1InitSmsig) {
        vds = s0[kB4SVds];
        vgs = s0[kB4SVgs];
        vbs = s0[kB4SVbs];
        vges = s0[kB4SVges];
        vgms = s0[kB4SVgms];
        vdbs = s0[kB4SVdbs];
        vsbs = s0[kB4SVsbs];
        vses = s0[kB4SVses];
        vdes = s0[kB4SVdes];
    } else if (mode & kM1InitTran) {
        vds = s1[kB4SVds];
        vgs = s1[kB4SVgs];
        vbs = s1[kB4SVbs];
        vges = s1[kB4SVges];
        vgms = s1[kB4SVgms];
        vdbs = s1[kB4SVdbs];
        vsbs = s1[kB4SVsbs];
        vses = s1[kB4SVses];
        vdes = s1[kB4SVdes];
    } else if ((mode & kM1InitJct) && !off) {
        vds = type * P[kB4IcVds];
        vgs = vges = vgms = type * P[kB4IcVgs];
        vbs = vdbs = vsbs = type * P[kB4IcVbs];
        if (vds > 0.0) {
            vdes = vds + 0.01;
            vses = -0.01;
        } else if (vds < 0.0) {
            vdes = vds - 0.01;
            vses = 0.01;
        } else {
            vdes = vses = 0.0;
        }
        if ((vds == 0.0) && (vgs == 0.0) && (vbs == 0.0) &&
            ((mode & (kM1Tran | kM1DcOp | kM1DcTranCurve)) || (!(mode & kM1Uic)))) {
            vds = 0.1;
            vdes = 0.11;
            vses = -0.01;
            vgs = vges = vgms = type * P[kB4Vth0] + 0.1;
            vbs = vdbs = vsbs = 0.0;
        }
    } else if ((mode & (kM1InitJct | kM1InitFix)) && off) {
        vds = vgs = vbs = vges = vgms = 0.0;
        vdbs = vsbs = vdes = vses = 0.0;
    } else {
        predicted = true;
        if (mode & kM1InitPred) {
            const double xfact = ic.delta / ic.delta_old1;
            s0[kB4SVds] = s1[kB4SVds];
            vds = (1.0 + xfact) * (s1[kB4SVds]) - (xfact * (s2[kB4SVds]));
            s0[kB4SVgs] = s1[kB4SVgs];
            vgs = (1.0 + xfact) * (s1[kB4SVgs]) - (xfact * (s2[kB4SVgs]));
            s0[kB4SVges] = s1[kB4SVges];
            vges = (1.0 + xfact) * (s1[kB4SVges]) - (xfact * (s2[kB4SVges]));
            s0[kB4SVgms] = s1[kB4SVgms];
            vgms = (1.0 + xfact) * (s1[kB4SVgms]) - (xfact * (s2[kB4SVgms]));
            s0[kB4SVbs] = s1[kB4SVbs];
            vbs = (1.0 + xfact) * (s1[kB4SVbs]) - (xfact * (s2[kB4SVbs]));
            s0[kB4SVbd] = s0[kB4SVbs] - s0[kB4SVds];
            s0[kB4SVdbs] = s1[kB4SVdbs];
            vdbs = (1.0 + xfact) * (s1[kB4SVdbs]) - (xfact * (s2[kB4SVdbs]));
            s0[kB4SVdbd] = s0[kB4SVdbs] - s0[kB4SVds];
            s0[kB4SVsbs] = s1[kB4SVsbs];
            vsbs = (1.0 + xfact) * (s1[kB4SVsbs]) - (xfact * (s2[kB4SVsbs]));
            s0[kB4SVses] = s1[kB4SVses];
            vses = (1.0 + xfact) * (s1[kB4SVses]) - (xfact * (s2[kB4SVses]));
            s0[kB4SVdes] = s1[kB4SVdes];
            vdes = (1.0 + xfact) * (s1[kB4SVdes]) - (xfact * (s2[kB4SVdes]));
            s0[kB4SQdef] = s1[kB4SQdef];
        } else {
            // No internal nodes: dNodePrime = dNode, gNodeExt = gNodeMid =
            // gNodePrime, dbNode = sbNode = bNodePrime.
            vds = type * (v[0] - v[2]);
            vgs = type * (v[1] - v[2]);
            vbs = type * (v[3] - v[2]);
            vges = type * (v[1] - v[2]);
            vgms = type * (v[1] - v[2]);
            vdbs = type * (v[3] - v[2]);
            vsbs = type * (v[3] - v[2]);
            vses = type * (v[2] - v[2]);
            vdes = type * (v[0] - v[2]);
        }
        const double vgdo = s0[kB4SVgs] - s0[kB4SVds];
        double vbd = vbs - vds;
        double vgd = vgs - vds;
        const double delvbd = vbd - s0[kB4SVbd];
        const double delvds = vds - s0[kB4SVds];
        const double delvgs = vgs - s0[kB4SVgs];
        const double delvbs = vbs - s0[kB4SVbs];
        const double delvgd = vgd - vgdo;
        // convergence prediction from the previous load's values
        if (rec[kB4RMode] >= 0) {
            Idtot = rec[kB4RCd] - rec[kB4RCbd];
            cdhat = Idtot - rec[kB4RGbd] * delvbd + rec[kB4RGmbs] * delvbs +
                    rec[kB4RGm] * delvgs + rec[kB4RGds] * delvds;
        } else {
            Idtot = rec[kB4RCd] + rec[kB4RCbd];
            cdhat = Idtot + rec[kB4RGbd] * delvbd + rec[kB4RGmbs] * delvbd +
                    rec[kB4RGm] * delvgd - rec[kB4RGds] * delvds;
        }
        Ibtot = rec[kB4RCbs] + rec[kB4RCbd];
        cbhat = (rec[kB4RMode] >= 0) ? Ibtot + rec[kB4RGbd] * delvbd + rec[kB4RGbs] * delvbs
                                      : Ibtot + rec[kB4RGbs] * delvbs + rec[kB4RGbd] * delvbd;
        // limiting (DEVfetlim / DEVlimvds / DEVpnjlim)
        const double von = rec[kB4RVon];
        if (s0[kB4SVds] >= 0.0) {
            vgs = m1_fetlim(vgs, s0[kB4SVgs], von);
            vds = vgs - vgd;
            vds = m1_limvds(vds, s0[kB4SVds]);
            vgd = vgs - vds;
        } else {
            vgd = m1_fetlim(vgd, vgdo, von);
            vds = vgs - vgd;
            vds = -m1_limvds(-vds, -(s0[kB4SVds]));
            vgs = vgd + vds;
        }
        if (vds >= 0.0) {
            vbs = m1_pnjlim(vbs, s0[kB4SVbs], kB4Vt0, P[kB4Vcrit], &Check);
        } else {
            vbd = m1_pnjlim(vbd, s0[kB4SVbd], kB4Vt0, P[kB4Vcrit], &Check);
            vbs = vbd + vds;
        }
    }
    (void)predicted;

    const double vbd = vbs - vds;
    const double vgd = vgs - vds;
    const double vgb = vgs - vbs;
    const double vdbd = vdbs - vds;
    const double vbs_jct = vbs;
    const double vbd_jct = vbd;

    // --- source / drain junction diodes, dioMod 1 (:675-785) ---
    const double Nvtms = P[kB4Vtm] * P[kB4NjS];
    double gbs, cbs, gbd, cbd;
    b4_junction_current(vbs_jct, P[kB4SatCurS], Nvtms, P[kB4VjsmFwd], P[kB4IVjsmFwd], gmin, &gbs,
                        &cbs);
    const double Nvtmd = P[kB4Vtm] * P[kB4NjD];
    b4_junction_current(vbd_jct, P[kB4SatCurD], Nvtmd, P[kB4VjdmFwd], P[kB4IVjdmFwd], gmin, &gbd,
                        &cbd);

    int dmode;
    double Vds, Vbs;
    if (vds >= 0.0) {
        dmode = 1;
        Vds = vds;
        Vbs = vbs;
    } else {
        dmode = -1;
        Vds = -vds;
        Vbs = vbd;
    }
    const double toxe = P[kB4Toxe];
    const double epssub = kB4Epssi;
    const double coxe = P[kB4Coxe];

    // --- Vbseff, Phis, Xdep (:1000-1040) ---
    const double vbsc = P[kB4Vbsc];
    double Vbseff, dVbseff_dVb;
    {
        const double T0 = Vbs - vbsc - 0.001;
        const double T1 = sqrt(T0 * T0 - 0.004 * vbsc);
        if (T0 >= 0.0) {
            Vbseff = vbsc + 0.5 * (T0 + T1);
            dVbseff_dVb = 0.5 * (1.0 + T0 / T1);
        } else {
            const double T2 = -0.002 / (T1 - T0);
            Vbseff = vbsc * (1.0 + T2);
            dVbseff_dVb = T2 * vbsc / T1;
        }
        const double T9 = 0.95 * P[kB4Phi];
        const double U0 = T9 - Vbseff - 0.001;
        const double U1 = sqrt(U0 * U0 + 0.004 * T9);
        Vbseff = T9 - 0.5 * (U0 + U1);
        dVbseff_dVb *= 0.5 * (1.0 + U0 / U1);
    }
    const double Phis = P[kB4Phi] - Vbseff;
    const double dPhis_dVb = -1.0;
    const double sqrtPhis = sqrt(Phis);
    const double dsqrtPhis_dVb = -0.5 / sqrtPhis;
    const double Xdep = P[kB4Xdep0] * sqrtPhis / P[kB4SqrtPhi];
    const double dXdep_dVb = (P[kB4Xdep0] / P[kB4SqrtPhi]) * dsqrtPhis_dVb;
    const double Leff = P[kB4Leff];
    const double Vtm = P[kB4Vtm];

    // --- threshold voltage (:1042-1160) ---
    double Vth, dVth_dVb, dVth_dVd, Theta0, dTheta0_dVb, Lpe_Vb, Vth_NarrowW;
    {
        double T3 = sqrt(Xdep);
        const double V0 = P[kB4Vbi] - P[kB4Phi];
        double T0 = P[kB4Dvt2] * Vbseff, T1, T2;
        if (T0 >= -0.5) {
            T1 = 1.0 + T0;
            T2 = P[kB4Dvt2];
        } else {
            const double T4 = 1.0 / (3.0 + 8.0 * T0);
            T1 = (1.0 + 3.0 * T0) * T4;
            T2 = P[kB4Dvt2] * T4 * T4;
        }
        const double lt1 = P[kB4Factor1] * T3 * T1;
        const double dlt1_dVb = P[kB4Factor1] * (0.5 / T3 * T1 * dXdep_dVb + T3 * T2);
        T0 = P[kB4Dvt2w] * Vbseff;
        if (T0 >= -0.5) {
            T1 = 1.0 + T0;
            T2 = P[kB4Dvt2w];
        } else {
            const double T4 = 1.0 / (3.0 + 8.0 * T0);
            T1 = (1.0 + 3.0 * T0) * T4;
            T2 = P[kB4Dvt2w] * T4 * T4;
        }
        const double ltw = P[kB4Factor1] * T3 * T1;
        const double dltw_dVb = P[kB4Factor1] * (0.5 / T3 * T1 * dXdep_dVb + T3 * T2);

        T0 = P[kB4Dvt1] * Leff / lt1;
        if (T0 < kB4ExpThreshold) {
            T1 = exp(T0);
            T2 = T1 - 1.0;
            T3 = T2 * T2;
            const double T4 = T3 + 2.0 * T1 * kB4MinExp;
            Theta0 = T1 / T4;
            const double dT1_dVb = -T0 * T1 * dlt1_dVb / lt1;
            dTheta0_dVb = dT1_dVb * (T4 - 2.0 * T1 * (T2 + kB4MinExp)) / T4 / T4;
        } else {
            Theta0 = 1.0 / (kB4MaxExp - 2.0);
            dTheta0_dVb = 0.0;
        }
        const double thetavth = P[kB4Dvt0] * Theta0;
        const double Delt_vth = thetavth * V0;
        const double dDelt_vth_dVb = P[kB4Dvt0] * dTheta0_dVb * V0;

        T0 = P[kB4Dvt1w] * P[kB4Weff] * Leff / ltw;
        double T5, dT5_dVb;
        if (T0 < kB4ExpThreshold) {
            T1 = exp(T0);
            T2 = T1 - 1.0;
            T3 = T2 * T2;
            const double T4 = T3 + 2.0 * T1 * kB4MinExp;
            T5 = T1 / T4;
            const double dT1_dVb = -T0 * T1 * dltw_dVb / ltw;
            dT5_dVb = dT1_dVb * (T4 - 2.0 * T1 * (T2 + kB4MinExp)) / T4 / T4;
        } else {
            T5 = 1.0 / (kB4MaxExp - 2.0);
            dT5_dVb = 0.0;
        }
        T0 = P[kB4Dvt0w] * T5;
        T2 = T0 * V0;
        const double dT2_dVb = P[kB4Dvt0w] * dT5_dVb * V0;

        const double TempRatio = P[kB4TempRatio];
        T0 = sqrt(1.0 + P[kB4Lpe0] / Leff);
        T1 = P[kB4K1ox] * (T0 - 1.0) * P[kB4SqrtPhi] +
             (P[kB4Kt1] + P[kB4Kt1l] / Leff + P[kB4Kt2] * Vbseff) * TempRatio;
        Vth_NarrowW = toxe * P[kB4Phi] / (P[kB4Weff] + P[kB4W0]);

        T3 = P[kB4Eta0] + P[kB4Etab] * Vbseff;
        double T4;
        if (T3 < 1.0e-4) {
            const double T9 = 1.0 / (3.0 - 2.0e4 * T3);
            T3 = (2.0e-4 - T3) * T9;
            T4 = T9 * T9;
        } else {
            T4 = 1.0;
        }
        const double dDIBL_Sft_dVd = T3 * P[kB4Theta0vb0];
        const double DIBL_Sft = dDIBL_Sft_dVd * Vds;

        Lpe_Vb = sqrt(1.0 + P[kB4Lpeb] / Leff);

        Vth = type * P[kB4Vth0] + (P[kB4K1ox] * sqrtPhis - P[kB4K1] * P[kB4SqrtPhi]) * Lpe_Vb -
              P[kB4K2ox] * Vbseff - Delt_vth - T2 + (P[kB4K3] + P[kB4K3b] * Vbseff) * Vth_NarrowW +
              T1 - DIBL_Sft;
        dVth_dVb = Lpe_Vb * P[kB4K1ox] * dsqrtPhis_dVb - P[kB4K2ox] - dDelt_vth_dVb - dT2_dVb +
                   P[kB4K3b] * Vth_NarrowW - P[kB4Etab] * Vds * P[kB4Theta0vb0] * T4 +
                   P[kB4Kt2] * TempRatio;
        dVth_dVd = -dDIBL_Sft_dVd;
    }

    // --- subthreshold swing n (:1162-1187) ---
    double n, dn_dVb, dn_dVd;
    {
        const double tmp1 = epssub / Xdep;
        const double tmp2 = P[kB4Nfactor] * tmp1;
        const double tmp3 = P[kB4Cdsc] + P[kB4Cdscb] * Vbseff + P[kB4Cdscd] * Vds;
        const double tmp4 = (tmp2 + tmp3 * Theta0 + P[kB4Cit]) / coxe;
        if (tmp4 >= -0.5) {
            n = 1.0 + tmp4;
            dn_dVb = (-tmp2 / Xdep * dXdep_dVb + tmp3 * dTheta0_dVb + P[kB4Cdscb] * Theta0) / coxe;
            dn_dVd = P[kB4Cdscd] * Theta0 / coxe;
        } else {
            double T0 = 1.0 / (3.0 + 8.0 * tmp4);
            n = (1.0 + 3.0 * tmp4) * T0;
            T0 *= T0;
            dn_dVb = (-tmp2 / Xdep * dXdep_dVb + tmp3 * dTheta0_dVb + P[kB4Cdscb] * Theta0) / coxe *
                     T0;
            dn_dVd = P[kB4Cdscd] * Theta0 / coxe * T0;
        }
    }
    const double von_new = Vth;

    // No poly depletion (NGATE = 0): Vgs_eff = vgs (or vgd in reverse mode).
    const double Vgs_eff = (dmode > 0) ? vgs : vgd;
    const double dVgs_eff_dVg = 1.0;
    const double Vgst = Vgs_eff - Vth;

    // --- Vgsteff (:1240-1300) ---
    double Vgsteff, dVgsteff_dVg, dVgsteff_dVd, dVgsteff_dVb;
    {
        const double mstar = P[kB4Mstar];
        double T0 = n * Vtm;
        double T1 = mstar * Vgst;
        double T2 = T1 / T0;
        double T10, dT10_dVg, dT10_dVd, dT10_dVb;
        if (T2 > kB4ExpThreshold) {
            T10 = T1;
            dT10_dVg = mstar * dVgs_eff_dVg;
            dT10_dVd = -dVth_dVd * mstar;
            dT10_dVb = -dVth_dVb * mstar;
        } else if (T2 < -kB4ExpThreshold) {
            T10 = Vtm * log(1.0 + kB4MinExp);
            dT10_dVg = 0.0;
            dT10_dVd = T10 * dn_dVd;
            dT10_dVb = T10 * dn_dVb;
            T10 *= n;
        } else {
            const double ExpVgst = exp(T2);
            const double T3 = Vtm * log(1.0 + ExpVgst);
            T10 = n * T3;
            dT10_dVg = mstar * ExpVgst / (1.0 + ExpVgst);
            dT10_dVb = T3 * dn_dVb - dT10_dVg * (dVth_dVb + Vgst * dn_dVb / n);
            dT10_dVd = T3 * dn_dVd - dT10_dVg * (dVth_dVd + Vgst * dn_dVd / n);
            dT10_dVg *= dVgs_eff_dVg;
        }
        T1 = P[kB4Voffcbn] - (1.0 - mstar) * Vgst;
        T2 = T1 / T0;
        double T9, dT9_dVg, dT9_dVd, dT9_dVb;
        if (T2 < -kB4ExpThreshold) {
            const double T3 = coxe * kB4MinExp / P[kB4Cdep0];
            T9 = mstar + T3 * n;
            dT9_dVg = 0.0;
            dT9_dVd = dn_dVd * T3;
            dT9_dVb = dn_dVb * T3;
        } else if (T2 > kB4ExpThreshold) {
            const double T3 = coxe * kB4MaxExp / P[kB4Cdep0];
            T9 = mstar + T3 * n;
            dT9_dVg = 0.0;
            dT9_dVd = dn_dVd * T3;
            dT9_dVb = dn_dVb * T3;
        } else {
            const double ExpVgst = exp(T2);
            const double T3 = coxe / P[kB4Cdep0];
            const double T4 = T3 * ExpVgst;
            const double T5 = T1 * T4 / T0;
            T9 = mstar + n * T4;
            dT9_dVg = T3 * (mstar - 1.0) * ExpVgst / Vtm;
            dT9_dVb = T4 * dn_dVb - dT9_dVg * dVth_dVb - T5 * dn_dVb;
            dT9_dVd = T4 * dn_dVd - dT9_dVg * dVth_dVd - T5 * dn_dVd;
            dT9_dVg *= dVgs_eff_dVg;
        }
        Vgsteff = T10 / T9;
        const double T11 = T9 * T9;
        dVgsteff_dVg = (T9 * dT10_dVg - T10 * dT9_dVg) / T11;
        dVgsteff_dVd = (T9 * dT10_dVd - T10 * dT9_dVd) / T11;
        dVgsteff_dVb = (T9 * dT10_dVb - T10 * dT9_dVb) / T11;
    }

    // --- effective width and Rds (:1302-1340, rdsMod 0) ---
    double Weff, dWeff_dVg, dWeff_dVb, Rds, dRds_dVg, dRds_dVb;
    double T9w = sqrtPhis - P[kB4SqrtPhi];
    {
        Weff = P[kB4Weff] - 2.0 * (P[kB4Dwg] * Vgsteff + P[kB4Dwb] * T9w);
        dWeff_dVg = -2.0 * P[kB4Dwg];
        dWeff_dVb = -2.0 * P[kB4Dwb] * dsqrtPhis_dVb;
        if (Weff < 2.0e-8) {
            double T0 = 1.0 / (6.0e-8 - 2.0 * Weff);
            Weff = 2.0e-8 * (4.0e-8 - Weff) * T0;
            T0 *= T0 * 4.0e-16;
            dWeff_dVg *= T0;
            dWeff_dVb *= T0;
        }
        const double T0 = 1.0 + P[kB4Prwg] * Vgsteff;
        const double dT0_dVg = -P[kB4Prwg] / T0 / T0;
        const double T1 = P[kB4Prwb] * T9w;
        const double dT1_dVb = P[kB4Prwb] * dsqrtPhis_dVb;
        const double T2 = 1.0 / T0 + T1;
        const double T3 = T2 + sqrt(T2 * T2 + 0.01);
        double dT3_dVg = 1.0 + T2 / (T3 - T2);
        const double dT3_dVb = dT3_dVg * dT1_dVb;
        dT3_dVg *= dT0_dVg;
        const double T4 = P[kB4Rds0] * 0.5;
        Rds = P[kB4Rdswmin] + T3 * T4;
        dRds_dVg = T4 * dT3_dVg;
        dRds_dVb = T4 * dT3_dVb;
    }

    // --- Abulk (:1342-1400) ---
    double Abulk, Abulk0, dAbulk_dVg, dAbulk_dVb, dAbulk0_dVb;
    {
        double T9 = 0.5 * P[kB4K1ox] * Lpe_Vb / sqrtPhis;
        const double T1 = T9 + P[kB4K2ox] - P[kB4K3b] * Vth_NarrowW;
        const double dT1_dVb = -T9 / sqrtPhis * dsqrtPhis_dVb;
        T9 = sqrt(P[kB4Xj] * Xdep);
        const double tmp1 = Leff + 2.0 * T9;
        const double T5 = Leff / tmp1;
        const double tmp2 = P[kB4A0] * T5;
        const double tmp3 = P[kB4Weff] + P[kB4B1];
        const double tmp4 = P[kB4B0] / tmp3;
        const double T2 = tmp2 + tmp4;
        const double dT2_dVb = -T9 / tmp1 / Xdep * dXdep_dVb;
        const double T6 = T5 * T5;
        const double T7 = T5 * T6;
        Abulk0 = 1.0 + T1 * T2;
        dAbulk0_dVb = T1 * tmp2 * dT2_dVb + T2 * dT1_dVb;
        const double T8 = P[kB4Ags] * P[kB4A0] * T7;
        dAbulk_dVg = -T1 * T8;
        Abulk = Abulk0 + dAbulk_dVg * Vgsteff;
        dAbulk_dVb = dAbulk0_dVb - T8 * Vgsteff * (dT1_dVb + 3.0 * T1 * dT2_dVb);
        if (Abulk0 < 0.1) {
            T9 = 1.0 / (3.0 - 20.0 * Abulk0);
            Abulk0 = (0.2 - Abulk0) * T9;
            dAbulk0_dVb *= T9 * T9;
        }
        if (Abulk < 0.1) {
            T9 = 1.0 / (3.0 - 20.0 * Abulk);
            Abulk = (0.2 - Abulk) * T9;
            const double T10 = T9 * T9;
            dAbulk_dVb *= T10;
            dAbulk_dVg *= T10;
        }
        const double T2k = P[kB4Keta] * Vbseff;
        double T0, dT0_dVb;
        if (T2k >= -0.9) {
            T0 = 1.0 / (1.0 + T2k);
            dT0_dVb = -P[kB4Keta] * T0 * T0;
        } else {
            const double T1k = 1.0 / (0.8 + T2k);
            T0 = (17.0 + 20.0 * T2k) * T1k;
            dT0_dVb = -P[kB4Keta] * T1k * T1k;
        }
        dAbulk_dVg *= T0;
        dAbulk_dVb = dAbulk_dVb * T0 + Abulk * dT0_dVb;
        dAbulk0_dVb = dAbulk0_dVb * T0 + Abulk0 * dT0_dVb;
        Abulk *= T0;
        Abulk0 *= T0;
    }

    // --- mobility, mobMod 0 (:1402-1420, 1497-1514) ---
    double ueff, dueff_dVg, dueff_dVd, dueff_dVb;
    {
        const double T14 = 0.0;
        const double T0 = Vgsteff + Vth + Vth - T14;
        const double T2 = P[kB4Ua] + P[kB4Uc] * Vbseff;
        const double T3 = T0 / toxe;
        const double T12 = sqrt(Vth * Vth + 0.0001);
        const double T9 = 1.0 / (Vgsteff + 2 * T12);
        const double T10 = T9 * toxe;
        const double T8 = P[kB4Ud] * T10 * T10 * Vth;
        const double T6 = T8 * Vth;
        const double T5 = T3 * (T2 + P[kB4Ub] * T3) + T6;
        const double T7 = -2.0 * T6 * T9;
        const double T11 = T7 * Vth / T12;
        double dDenomi_dVg = (T2 + 2.0 * P[kB4Ub] * T3) / toxe;
        const double T13 = 2.0 * (dDenomi_dVg + T11 + T8);
        double dDenomi_dVd = T13 * dVth_dVd;
        double dDenomi_dVb = T13 * dVth_dVb + P[kB4Uc] * T3;
        dDenomi_dVg += T7;
        double Denomi;
        if (T5 >= -0.8) {
            Denomi = 1.0 + T5;
        } else {
            double T9d = 1.0 / (7.0 + 10.0 * T5);
            Denomi = (0.6 + T5) * T9d;
            T9d *= T9d;
            dDenomi_dVg *= T9d;
            dDenomi_dVd *= T9d;
            dDenomi_dVb *= T9d;
        }
        ueff = P[kB4U0temp] / Denomi;
        const double T9u = -ueff / Denomi;
        dueff_dVg = T9u * dDenomi_dVg;
        dueff_dVd = T9u * dDenomi_dVd;
        dueff_dVb = T9u * dDenomi_dVb;
    }

    // --- Vdsat (:1516-1620) ---
    const double WVCox = Weff * P[kB4Vsattemp] * coxe;
    const double WVCoxRds = WVCox * Rds;
    double Esat = 2.0 * P[kB4Vsattemp] / ueff;
    double EsatL = Esat * Leff;
    double dEsatL_dVg, dEsatL_dVd, dEsatL_dVb;
    {
        const double T0 = -EsatL / ueff;
        dEsatL_dVg = T0 * dueff_dVg;
        dEsatL_dVd = T0 * dueff_dVd;
        dEsatL_dVb = T0 * dueff_dVb;
    }
    double Lambda, dLambda_dVg;
    {
        const double a1 = P[kB4A1];
        if (a1 == 0.0) {
            Lambda = P[kB4A2];
            dLambda_dVg = 0.0;
        } else if (a1 > 0.0) {
            const double T0 = 1.0 - P[kB4A2];
            const double T1 = T0 - P[kB4A1] * Vgsteff - 0.0001;
            const double T2 = sqrt(T1 * T1 + 0.0004 * T0);
            Lambda = P[kB4A2] + T0 - 0.5 * (T1 + T2);
            dLambda_dVg = 0.5 * P[kB4A1] * (1.0 + T1 / T2);
        } else {
            const double T1 = P[kB4A2] + P[kB4A1] * Vgsteff - 0.0001;
            const double T2 = sqrt(T1 * T1 + 0.0004 * P[kB4A2]);
            Lambda = 0.5 * (T1 + T2);
            dLambda_dVg = 0.5 * P[kB4A1] * (1.0 + T1 / T2);
        }
    }
    const double Vgst2Vtm = Vgsteff + 2.0 * Vtm;
    double tmp1v, tmp2v, tmp3v;
    if (Rds > 0) {
        tmp2v = dRds_dVg / Rds + dWeff_dVg / Weff;
        tmp3v = dRds_dVb / Rds + dWeff_dVb / Weff;
    } else {
        tmp2v = dWeff_dVg / Weff;
        tmp3v = dWeff_dVb / Weff;
    }
    double Vdsat, dVdsat_dVg, dVdsat_dVd, dVdsat_dVb;
    if ((Rds == 0.0) && (Lambda == 1.0)) {
        const double T0 = 1.0 / (Abulk * EsatL + Vgst2Vtm);
        tmp1v = 0.0;
        const double T1 = T0 * T0;
        const double T2 = Vgst2Vtm * T0;
        const double T3 = EsatL * Vgst2Vtm;
        Vdsat = T3 * T0;
        const double dT0_dVg = -(Abulk * dEsatL_dVg + EsatL * dAbulk_dVg + 1.0) * T1;
        const double dT0_dVd = -(Abulk * dEsatL_dVd) * T1;
        const double dT0_dVb = -(Abulk * dEsatL_dVb + dAbulk_dVb * EsatL) * T1;
        dVdsat_dVg = T3 * dT0_dVg + T2 * dEsatL_dVg + EsatL * T0;
        dVdsat_dVd = T3 * dT0_dVd + T2 * dEsatL_dVd;
        dVdsat_dVb = T3 * dT0_dVb + T2 * dEsatL_dVb;
    } else {
        tmp1v = dLambda_dVg / (Lambda * Lambda);
        const double T9 = Abulk * WVCoxRds;
        const double T8 = Abulk * T9;
        const double T7 = Vgst2Vtm * T9;
        const double T6 = Vgst2Vtm * WVCoxRds;
        const double T0 = 2.0 * Abulk * (T9 - 1.0 + 1.0 / Lambda);
        const double dT0_dVg = 2.0 * (T8 * tmp2v - Abulk * tmp1v +
                                      (2.0 * T9 + 1.0 / Lambda - 1.0) * dAbulk_dVg);
        const double dT0_dVb = 2.0 * (T8 * (2.0 / Abulk * dAbulk_dVb + tmp3v) +
                                      (1.0 / Lambda - 1.0) * dAbulk_dVb);
        const double dT0_dVd = 0.0;
        const double T1 = Vgst2Vtm * (2.0 / Lambda - 1.0) + Abulk * EsatL + 3.0 * T7;
        const double dT1_dVg = (2.0 / Lambda - 1.0) - 2.0 * Vgst2Vtm * tmp1v + Abulk * dEsatL_dVg +
                               EsatL * dAbulk_dVg + 3.0 * (T9 + T7 * tmp2v + T6 * dAbulk_dVg);
        const double dT1_dVb =
            Abulk * dEsatL_dVb + EsatL * dAbulk_dVb + 3.0 * (T6 * dAbulk_dVb + T7 * tmp3v);
        const double dT1_dVd = Abulk * dEsatL_dVd;
        const double T2 = Vgst2Vtm * (EsatL + 2.0 * T6);
        const double dT2_dVg = EsatL + Vgst2Vtm * dEsatL_dVg + T6 * (4.0 + 2.0 * Vgst2Vtm * tmp2v);
        const double dT2_dVb = Vgst2Vtm * (dEsatL_dVb + 2.0 * T6 * tmp3v);
        const double dT2_dVd = Vgst2Vtm * dEsatL_dVd;
        const double T3 = sqrt(T1 * T1 - 2.0 * T0 * T2);
        Vdsat = (T1 - T3) / T0;
        dVdsat_dVg = (dT1_dVg - (T1 * dT1_dVg - dT0_dVg * T2 - T0 * dT2_dVg) / T3 -
                      Vdsat * dT0_dVg) / T0;
        dVdsat_dVb = (dT1_dVb - (T1 * dT1_dVb - dT0_dVb * T2 - T0 * dT2_dVb) / T3 -
                      Vdsat * dT0_dVb) / T0;
        dVdsat_dVd = (dT1_dVd - (T1 * dT1_dVd - T0 * dT2_dVd) / T3) / T0;
        (void)dT0_dVd;
    }

    // --- Vdseff (:1622-1660) ---
    double Vdseff, dVdseff_dVg, dVdseff_dVd, dVdseff_dVb;
    {
        const double T1 = Vdsat - Vds - P[kB4Delta];
        const double dT1_dVg = dVdsat_dVg;
        const double dT1_dVd = dVdsat_dVd - 1.0;
        const double dT1_dVb = dVdsat_dVb;
        const double T2 = sqrt(T1 * T1 + 4.0 * P[kB4Delta] * Vdsat);
        const double T0 = T1 / T2;
        const double T9 = 2.0 * P[kB4Delta];
        const double T3 = T9 / T2;
        const double dT2_dVg = T0 * dT1_dVg + T3 * dVdsat_dVg;
        const double dT2_dVd = T0 * dT1_dVd + T3 * dVdsat_dVd;
        const double dT2_dVb = T0 * dT1_dVb + T3 * dVdsat_dVb;
        if (T1 >= 0.0) {
            Vdseff = Vdsat - 0.5 * (T1 + T2);
            dVdseff_dVg = dVdsat_dVg - 0.5 * (dT1_dVg + dT2_dVg);
            dVdseff_dVd = dVdsat_dVd - 0.5 * (dT1_dVd + dT2_dVd);
            dVdseff_dVb = dVdsat_dVb - 0.5 * (dT1_dVb + dT2_dVb);
        } else {
            const double T4 = T9 / (T2 - T1);
            const double T5 = 1.0 - T4;
            const double T6 = Vdsat * T4 / (T2 - T1);
            Vdseff = Vdsat * T5;
            dVdseff_dVg = dVdsat_dVg * T5 + T6 * (dT2_dVg - dT1_dVg);
            dVdseff_dVd = dVdsat_dVd * T5 + T6 * (dT2_dVd - dT1_dVd);
            dVdseff_dVb = dVdsat_dVb * T5 + T6 * (dT2_dVb - dT1_dVb);
        }
        if (Vds == 0.0) {
            Vdseff = 0.0;
            dVdseff_dVg = 0.0;
            dVdseff_dVb = 0.0;
        }
        if (Vdseff > Vds) Vdseff = Vds;
    }
    const double diffVds = Vds - Vdseff;

    // --- Vasat (:1700-1730) ---
    double Vasat, dVasat_dVg, dVasat_dVd, dVasat_dVb;
    {
        const double tmp4 = 1.0 - 0.5 * Abulk * Vdsat / Vgst2Vtm;
        double T9 = WVCoxRds * Vgsteff;
        const double T8 = T9 / Vgst2Vtm;
        const double T0 = EsatL + Vdsat + 2.0 * T9 * tmp4;
        const double T7 = 2.0 * WVCoxRds * tmp4;
        const double dT0_dVg = dEsatL_dVg + dVdsat_dVg + T7 * (1.0 + tmp2v * Vgsteff) -
                               T8 * (Abulk * dVdsat_dVg - Abulk * Vdsat / Vgst2Vtm +
                                     Vdsat * dAbulk_dVg);
        const double dT0_dVb = dEsatL_dVb + dVdsat_dVb + T7 * tmp3v * Vgsteff -
                               T8 * (dAbulk_dVb * Vdsat + Abulk * dVdsat_dVb);
        const double dT0_dVd = dEsatL_dVd + dVdsat_dVd - T8 * Abulk * dVdsat_dVd;
        T9 = WVCoxRds * Abulk;
        const double T1 = 2.0 / Lambda - 1.0 + T9;
        const double dT1_dVg = -2.0 * tmp1v + WVCoxRds * (Abulk * tmp2v + dAbulk_dVg);
        const double dT1_dVb = dAbulk_dVb * WVCoxRds + T9 * tmp3v;
        Vasat = T0 / T1;
        dVasat_dVg = (dT0_dVg - Vasat * dT1_dVg) / T1;
        dVasat_dVb = (dT0_dVb - Vasat * dT1_dVb) / T1;
        dVasat_dVd = dT0_dVd / T1;
    }

    // --- Idl (:1732-1790) ---
    double Idl, dIdl_dVg, dIdl_dVd, dIdl_dVb, Coxeff_iv;
    {
        const double tmp1 = P[kB4Vtfbphi2];
        const double tmp2 = 2.0e8 * P[kB4Toxp];
        const double dT0_dVg = 1.0 / tmp2;
        double T0 = (Vgsteff + tmp1) * dT0_dVg;
        const double tmp3 = exp(P[kB4Bdos] * 0.7 * log(T0));
        double T1 = 1.0 + tmp3;
        double T2 = P[kB4Bdos] * 0.7 * tmp3 / T0;
        const double Tcen = P[kB4Ados] * 1.9e-9 / T1;
        const double dTcen_dVg = -Tcen * T2 * dT0_dVg / T1;
        const double Coxeff = epssub * P[kB4Coxp] / (epssub + P[kB4Coxp] * Tcen);
        Coxeff_iv = Coxeff;
        const double dCoxeff_dVg = -Coxeff * Coxeff * dTcen_dVg / epssub;
        const double CoxeffWovL = Coxeff * Weff / Leff;
        const double beta = ueff * CoxeffWovL;
        const double T3 = ueff / Leff;
        const double dbeta_dVg = CoxeffWovL * dueff_dVg + T3 * (Weff * dCoxeff_dVg + Coxeff * dWeff_dVg);
        const double dbeta_dVd = CoxeffWovL * dueff_dVd;
        const double dbeta_dVb = CoxeffWovL * dueff_dVb + T3 * Coxeff * dWeff_dVb;
        const double AbovVgst2Vtm = Abulk / Vgst2Vtm;
        T0 = 1.0 - 0.5 * Vdseff * AbovVgst2Vtm;
        const double dT0g = -0.5 * (Abulk * dVdseff_dVg - Abulk * Vdseff / Vgst2Vtm +
                                    Vdseff * dAbulk_dVg) / Vgst2Vtm;
        const double dT0d = -0.5 * Abulk * dVdseff_dVd / Vgst2Vtm;
        const double dT0b = -0.5 * (Abulk * dVdseff_dVb + dAbulk_dVb * Vdseff) / Vgst2Vtm;
        const double fgche1 = Vgsteff * T0;
        const double dfgche1_dVg = Vgsteff * dT0g + T0;
        const double dfgche1_dVd = Vgsteff * dT0d;
        const double dfgche1_dVb = Vgsteff * dT0b;
        const double T9 = Vdseff / EsatL;
        const double fgche2 = 1.0 + T9;
        const double dfgche2_dVg = (dVdseff_dVg - T9 * dEsatL_dVg) / EsatL;
        const double dfgche2_dVd = (dVdseff_dVd - T9 * dEsatL_dVd) / EsatL;
        const double dfgche2_dVb = (dVdseff_dVb - T9 * dEsatL_dVb) / EsatL;
        const double gche = beta * fgche1 / fgche2;
        const double dgche_dVg = (beta * dfgche1_dVg + fgche1 * dbeta_dVg - gche * dfgche2_dVg) / fgche2;
        const double dgche_dVd = (beta * dfgche1_dVd + fgche1 * dbeta_dVd - gche * dfgche2_dVd) / fgche2;
        const double dgche_dVb = (beta * dfgche1_dVb + fgche1 * dbeta_dVb - gche * dfgche2_dVb) / fgche2;
        T0 = 1.0 + gche * Rds;
        Idl = gche / T0;
        T1 = (1.0 - Idl * Rds) / T0;
        T2 = Idl * Idl;
        dIdl_dVg = T1 * dgche_dVg - T2 * dRds_dVg;
        dIdl_dVd = T1 * dgche_dVd;
        dIdl_dVb = T1 * dgche_dVb - T2 * dRds_dVb;
    }
    (void)Coxeff_iv;

    // FPROUT = 0 and PVAG = 0: FP = 1, PvagTerm = 1 + 0 (:1792-1820).
    const double FP = 1.0, dFP_dVg = 0.0;
    double PvagTerm, dPvagTerm_dVg, dPvagTerm_dVb, dPvagTerm_dVd;
    {
        const double T8 = 0.0 / EsatL;
        const double T9 = T8 * Vgsteff;
        PvagTerm = 1.0 + T9;
        dPvagTerm_dVg = T8 * (1.0 - Vgsteff * dEsatL_dVg / EsatL);
        dPvagTerm_dVb = -T9 * dEsatL_dVb / EsatL;
        dPvagTerm_dVd = -T9 * dEsatL_dVd / EsatL;
    }

    // --- VACLM (:1822-1850) ---
    double Cclm, dCclm_dVg, dCclm_dVd, dCclm_dVb, VACLM, dVACLM_dVg, dVACLM_dVd, dVACLM_dVb;
    if ((P[kB4Pclm] > kB4MinExp) && (diffVds > 1.0e-10)) {
        const double T0 = 1.0 + Rds * Idl;
        const double dT0_dVg = dRds_dVg * Idl + Rds * dIdl_dVg;
        const double dT0_dVd = Rds * dIdl_dVd;
        const double dT0_dVb = dRds_dVb * Idl + Rds * dIdl_dVb;
        const double T2 = Vdsat / Esat;
        const double T1 = Leff + T2;
        const double dT1_dVg = (dVdsat_dVg - T2 * dEsatL_dVg / Leff) / Esat;
        const double dT1_dVd = (dVdsat_dVd - T2 * dEsatL_dVd / Leff) / Esat;
        const double dT1_dVb = (dVdsat_dVb - T2 * dEsatL_dVb / Leff) / Esat;
        Cclm = FP * PvagTerm * T0 * T1 / (P[kB4Pclm] * P[kB4Litl]);
        dCclm_dVg = Cclm * (dFP_dVg / FP + dPvagTerm_dVg / PvagTerm + dT0_dVg / T0 + dT1_dVg / T1);
        dCclm_dVb = Cclm * (dPvagTerm_dVb / PvagTerm + dT0_dVb / T0 + dT1_dVb / T1);
        dCclm_dVd = Cclm * (dPvagTerm_dVd / PvagTerm + dT0_dVd / T0 + dT1_dVd / T1);
        VACLM = Cclm * diffVds;
        dVACLM_dVg = dCclm_dVg * diffVds - dVdseff_dVg * Cclm;
        dVACLM_dVb = dCclm_dVb * diffVds - dVdseff_dVb * Cclm;
        dVACLM_dVd = dCclm_dVd * diffVds + (1.0 - dVdseff_dVd) * Cclm;
    } else {
        VACLM = Cclm = kB4MaxExp;
        dVACLM_dVd = dVACLM_dVg = dVACLM_dVb = 0.0;
        dCclm_dVd = dCclm_dVg = dCclm_dVb = 0.0;
    }

    // --- VADIBL (:1852-1898) ---
    double VADIBL, dVADIBL_dVg, dVADIBL_dVd, dVADIBL_dVb;
    if (P[kB4ThetaRout] > kB4MinExp) {
        const double T8 = Abulk * Vdsat;
        const double T0 = Vgst2Vtm * T8;
        const double dT0_dVg = Vgst2Vtm * Abulk * dVdsat_dVg + T8 + Vgst2Vtm * Vdsat * dAbulk_dVg;
        const double dT0_dVb = Vgst2Vtm * (dAbulk_dVb * Vdsat + Abulk * dVdsat_dVb);
        const double dT0_dVd = Vgst2Vtm * Abulk * dVdsat_dVd;
        const double T1 = Vgst2Vtm + T8;
        const double dT1_dVg = 1.0 + Abulk * dVdsat_dVg + Vdsat * dAbulk_dVg;
        const double dT1_dVb = Abulk * dVdsat_dVb + dAbulk_dVb * Vdsat;
        const double dT1_dVd = Abulk * dVdsat_dVd;
        const double T9 = T1 * T1;
        const double T2 = P[kB4ThetaRout];
        VADIBL = (Vgst2Vtm - T0 / T1) / T2;
        dVADIBL_dVg = (1.0 - dT0_dVg / T1 + T0 * dT1_dVg / T9) / T2;
        dVADIBL_dVb = (-dT0_dVb / T1 + T0 * dT1_dVb / T9) / T2;
        dVADIBL_dVd = (-dT0_dVd / T1 + T0 * dT1_dVd / T9) / T2;
        const double T7 = P[kB4Pdiblb] * Vbseff;
        if (T7 >= -0.9) {
            const double T3 = 1.0 / (1.0 + T7);
            VADIBL *= T3;
            dVADIBL_dVg *= T3;
            dVADIBL_dVb = (dVADIBL_dVb - VADIBL * P[kB4Pdiblb]) * T3;
            dVADIBL_dVd *= T3;
        } else {
            const double T4 = 1.0 / (0.8 + T7);
            const double T3 = (17.0 + 20.0 * T7) * T4;
            dVADIBL_dVg *= T3;
            dVADIBL_dVb = dVADIBL_dVb * T3 - VADIBL * P[kB4Pdiblb] * T4 * T4;
            dVADIBL_dVd *= T3;
            VADIBL *= T3;
        }
        dVADIBL_dVg = dVADIBL_dVg * PvagTerm + VADIBL * dPvagTerm_dVg;
        dVADIBL_dVb = dVADIBL_dVb * PvagTerm + VADIBL * dPvagTerm_dVb;
        dVADIBL_dVd = dVADIBL_dVd * PvagTerm + VADIBL * dPvagTerm_dVd;
        VADIBL *= PvagTerm;
    } else {
        VADIBL = kB4MaxExp;
        dVADIBL_dVd = dVADIBL_dVg = dVADIBL_dVb = 0.0;
    }

    // --- Va, VADITS (PDITS = 0), VASCBE (:1900-1950) ---
    const double Va = Vasat + VACLM;
    const double dVa_dVg = dVasat_dVg + dVACLM_dVg;
    const double dVa_dVb = dVasat_dVb + dVACLM_dVb;
    const double dVa_dVd = dVasat_dVd + dVACLM_dVd;
    const double VADITS = kB4MaxExp, dVADITS_dVg = 0.0, dVADITS_dVd = 0.0;
    double VASCBE, dVASCBE_dVg, dVASCBE_dVd, dVASCBE_dVb;
    if ((P[kB4Pscbe2] > 0.0) && (P[kB4Pscbe1] >= 0.0)) {
        if (diffVds > P[kB4Pscbe1] * P[kB4Litl] / kB4ExpThreshold) {
            const double T0 = P[kB4Pscbe1] * P[kB4Litl] / diffVds;
            VASCBE = Leff * exp(T0) / P[kB4Pscbe2];
            const double T1 = T0 * VASCBE / diffVds;
            dVASCBE_dVg = T1 * dVdseff_dVg;
            dVASCBE_dVd = -T1 * (1.0 - dVdseff_dVd);
            dVASCBE_dVb = T1 * dVdseff_dVb;
        } else {
            VASCBE = kB4MaxExp * Leff / P[kB4Pscbe2];
            dVASCBE_dVg = dVASCBE_dVd = dVASCBE_dVb = 0.0;
        }
    } else {
        VASCBE = kB4MaxExp;
        dVASCBE_dVg = dVASCBE_dVd = dVASCBE_dVb = 0.0;
    }

    // --- Ids with DIBL, DITS, CLM, SCBE (:1952-2040) ---
    double Ids, Gm, Gds, Gmb, cdrain;
    {
        double T9 = diffVds / VADIBL;
        double T0 = 1.0 + T9;
        double Idsa = Idl * T0;
        double dIdsa_dVg = T0 * dIdl_dVg - Idl * (dVdseff_dVg + T9 * dVADIBL_dVg) / VADIBL;
        double dIdsa_dVd = T0 * dIdl_dVd + Idl * (1.0 - dVdseff_dVd - T9 * dVADIBL_dVd) / VADIBL;
        double dIdsa_dVb = T0 * dIdl_dVb - Idl * (dVdseff_dVb + T9 * dVADIBL_dVb) / VADIBL;

        T9 = diffVds / VADITS;
        T0 = 1.0 + T9;
        dIdsa_dVg = T0 * dIdsa_dVg - Idsa * (dVdseff_dVg + T9 * dVADITS_dVg) / VADITS;
        dIdsa_dVd = T0 * dIdsa_dVd + Idsa * (1.0 - dVdseff_dVd - T9 * dVADITS_dVd) / VADITS;
        dIdsa_dVb = T0 * dIdsa_dVb - Idsa * dVdseff_dVb / VADITS;
        Idsa *= T0;

        T0 = log(Va / Vasat);
        const double dT0_dVg = dVa_dVg / Va - dVasat_dVg / Vasat;
        const double dT0_dVb = dVa_dVb / Va - dVasat_dVb / Vasat;
        const double dT0_dVd = dVa_dVd / Va - dVasat_dVd / Vasat;
        const double T1 = T0 / Cclm;
        T9 = 1.0 + T1;
        const double dT9_dVg = (dT0_dVg - T1 * dCclm_dVg) / Cclm;
        const double dT9_dVb = (dT0_dVb - T1 * dCclm_dVb) / Cclm;
        const double dT9_dVd = (dT0_dVd - T1 * dCclm_dVd) / Cclm;
        dIdsa_dVg = dIdsa_dVg * T9 + Idsa * dT9_dVg;
        dIdsa_dVb = dIdsa_dVb * T9 + Idsa * dT9_dVb;
        dIdsa_dVd = dIdsa_dVd * T9 + Idsa * dT9_dVd;
        Idsa *= T9;

        // no substrate current (ALPHA0 = ALPHA1 = 0)
        T9 = diffVds / VASCBE;
        T0 = 1.0 + T9;
        Ids = Idsa * T0;
        Gm = T0 * dIdsa_dVg - Idsa * (dVdseff_dVg + T9 * dVASCBE_dVg) / VASCBE;
        Gds = T0 * dIdsa_dVd + Idsa * (1.0 - dVdseff_dVd - T9 * dVASCBE_dVd) / VASCBE;
        Gmb = T0 * dIdsa_dVb - Idsa * (dVdseff_dVb + T9 * dVASCBE_dVb) / VASCBE;
        const double tmp1 = Gds + Gm * dVgsteff_dVd;
        const double tmp2 = Gmb + Gm * dVgsteff_dVb;
        const double tmp3 = Gm;
        Gm = (Ids * dVdseff_dVg + Vdseff * tmp3) * dVgsteff_dVg;
        Gds = Ids * (dVdseff_dVd + dVdseff_dVg * dVgsteff_dVd) + Vdseff * tmp1;
        Gmb = (Ids * (dVdseff_dVb + dVdseff_dVg * dVgsteff_dVb) + Vdseff * tmp2) * dVbseff_dVb;
        cdrain = Ids * Vdseff;
    }
    const double gds = Gds, gm = Gm, gmbs = Gmb;

    // --- C-V (:2906-3842), capMod 2 ---
    double qgate = 0.0, qbulk = 0.0, qdrn = 0.0, qsrc = 0.0;
    double cggb = 0.0, cgsb = 0.0, cgdb = 0.0, cdgb = 0.0, cdsb = 0.0, cddb = 0.0, cbgb = 0.0,
           cbsb = 0.0, cbdb = 0.0;
    if (charge && !(P[kB4Xpart] < 0)) {
        double VbseffCV, dVbseffCV_dVb;
        if (Vbseff < 0.0) {
            VbseffCV = Vbseff;
            dVbseffCV_dVb = 1.0;
        } else {
            VbseffCV = P[kB4Phi] - Phis;
            dVbseffCV_dVb = -dPhis_dVb;
        }
        const double CoxWL = coxe * P[kB4WeffCV] * P[kB4LeffCV] * 1.0;
        // VgsteffCV (cvchargeMod 0)
        double VgsteffC, dVgC_dVg, dVgC_dVd, dVgC_dVb;
        {
            const double noff = n * P[kB4Noff];
            const double dnoff_dVd = P[kB4Noff] * dn_dVd;
            const double dnoff_dVb = P[kB4Noff] * dn_dVb;
            const double T0 = Vtm * noff;
            const double voffcv = P[kB4Voffcv];
            const double VgstNVt = (Vgst - voffcv) / T0;
            if (VgstNVt > kB4ExpThreshold) {
                VgsteffC = Vgst - voffcv;
                dVgC_dVg = dVgs_eff_dVg;
                dVgC_dVd = -dVth_dVd;
                dVgC_dVb = -dVth_dVb;
            } else if (VgstNVt < -kB4ExpThreshold) {
                VgsteffC = T0 * log(1.0 + kB4MinExp);
                dVgC_dVg = 0.0;
                dVgC_dVd = VgsteffC / noff;
                dVgC_dVb = dVgC_dVd * dnoff_dVb;
                dVgC_dVd *= dnoff_dVd;
            } else {
                const double ExpVgst = exp(VgstNVt);
                VgsteffC = T0 * log(1.0 + ExpVgst);
                dVgC_dVg = ExpVgst / (1.0 + ExpVgst);
                dVgC_dVd = -dVgC_dVg * (dVth_dVd + (Vgst - voffcv) / noff * dnoff_dVd) +
                           VgsteffC / noff * dnoff_dVd;
                dVgC_dVb = -dVgC_dVg * (dVth_dVb + (Vgst - voffcv) / noff * dnoff_dVb) +
                           VgsteffC / noff * dnoff_dVb;
                dVgC_dVg *= dVgs_eff_dVg;
            }
        }
        // charge-thickness model
        const double vfbzb = P[kB4Vfbzb];
        double V3 = vfbzb - Vgs_eff + VbseffCV - kB4Delta3;
        double T0 = (vfbzb <= 0.0) ? sqrt(V3 * V3 - 4.0 * kB4Delta3 * vfbzb)
                                   : sqrt(V3 * V3 + 4.0 * kB4Delta3 * vfbzb);
        double T1 = 0.5 * (1.0 + V3 / T0);
        const double Vfbeff = vfbzb - 0.5 * (V3 + T0);
        const double dVfbeff_dVg = T1 * dVgs_eff_dVg;
        const double dVfbeff_dVb = -T1 * dVbseffCV_dVb;

        const double Cox = P[kB4Coxp];
        double Tox = 1.0e8 * P[kB4Toxp];
        T0 = (Vgs_eff - VbseffCV - vfbzb) / Tox;
        const double dT0_dVg = dVgs_eff_dVg / Tox;
        const double dT0_dVb = -dVbseffCV_dVb / Tox;
        double tmp = T0 * P[kB4Acde];
        double Tcen, dTcen_dVg, dTcen_dVb;
        if ((-kB4ExpThreshold < tmp) && (tmp < kB4ExpThreshold)) {
            Tcen = P[kB4Ldeb] * exp(tmp);
            dTcen_dVg = P[kB4Acde] * Tcen;
            dTcen_dVb = dTcen_dVg * dT0_dVb;
            dTcen_dVg *= dT0_dVg;
        } else if (tmp <= -kB4ExpThreshold) {
            Tcen = P[kB4Ldeb] * kB4MinExp;
            dTcen_dVg = dTcen_dVb = 0.0;
        } else {
            Tcen = P[kB4Ldeb] * kB4MaxExp;
            dTcen_dVg = dTcen_dVb = 0.0;
        }
        const double LINK = 1.0e-3 * P[kB4Toxp];
        V3 = P[kB4Ldeb] - Tcen - LINK;
        const double V4 = sqrt(V3 * V3 + 4.0 * LINK * P[kB4Ldeb]);
        Tcen = P[kB4Ldeb] - 0.5 * (V3 + V4);
        T1 = 0.5 * (1.0 + V3 / V4);
        dTcen_dVg *= T1;
        dTcen_dVb *= T1;

        double Ccen = epssub / Tcen;
        double T2 = Cox / (Cox + Ccen);
        double Coxeff = T2 * Ccen;
        double T3 = -Ccen / Tcen;
        double dCoxeff_dVg = T2 * T2 * T3;
        double dCoxeff_dVb = dCoxeff_dVg * dTcen_dVb;
        dCoxeff_dVg *= dTcen_dVg;
        double CoxWLcen = CoxWL * Coxeff / coxe;

        const double Qac0 = CoxWLcen * (Vfbeff - vfbzb);
        double QovCox = Qac0 / Coxeff;
        const double dQac0_dVg = CoxWLcen * dVfbeff_dVg + QovCox * dCoxeff_dVg;
        const double dQac0_dVb = CoxWLcen * dVfbeff_dVb + QovCox * dCoxeff_dVb;

        T0 = 0.5 * P[kB4K1ox];
        T3 = Vgs_eff - Vfbeff - VbseffCV - VgsteffC;
        if (P[kB4K1ox] == 0.0) {
            T1 = 0.0;
            T2 = 0.0;
        } else if (T3 < 0.0) {
            T1 = T0 + T3 / P[kB4K1ox];
            T2 = CoxWLcen;
        } else {
            T1 = sqrt(T0 * T0 + T3);
            T2 = CoxWLcen * T0 / T1;
        }
        const double Qsub0 = CoxWLcen * P[kB4K1ox] * (T1 - T0);
        QovCox = Qsub0 / Coxeff;
        const double dQsub0_dVg = T2 * (dVgs_eff_dVg - dVfbeff_dVg - dVgC_dVg) + QovCox * dCoxeff_dVg;
        const double dQsub0_dVd = -T2 * dVgC_dVd;
        const double dQsub0_dVb =
            -T2 * (dVfbeff_dVb + dVbseffCV_dVb + dVgC_dVb) + QovCox * dCoxeff_dVb;

        double Denomi;
        if (P[kB4K1ox] <= 0.0) {
            Denomi = 0.25 * P[kB4Moin] * Vtm;
            T0 = 0.5 * P[kB4SqrtPhi];
        } else {
            Denomi = P[kB4Moin] * Vtm * P[kB4K1ox] * P[kB4K1ox];
            T0 = P[kB4K1ox] * P[kB4SqrtPhi];
        }
        T1 = 2.0 * T0 + VgsteffC;
        const double DeltaPhi = Vtm * log(1.0 + T1 * VgsteffC / Denomi);
        const double dDeltaPhi_dVg = 2.0 * Vtm * (T1 - T0) / (Denomi + T1 * VgsteffC);

        T0 = VgsteffC - DeltaPhi - 0.001;
        const double dT0g = 1.0 - dDeltaPhi_dVg;
        T1 = sqrt(T0 * T0 + VgsteffC * 0.004);
        const double VgDP = 0.5 * (T0 + T1);
        const double dVgDP_dVg = 0.5 * (dT0g + (T0 * dT0g + 0.002) / T1);

        Tox += Tox;
        T0 = (VgsteffC + P[kB4Vtfbphi2]) / Tox;
        tmp = exp(P[kB4Bdos] * 0.7 * log(T0));
        T1 = 1.0 + tmp;
        T2 = P[kB4Bdos] * 0.7 * tmp / (T0 * Tox);
        Tcen = P[kB4Ados] * 1.9e-9 / T1;
        dTcen_dVg = -Tcen * T2 / T1;
        const double dTcen_dVd = dTcen_dVg * dVgC_dVd;
        dTcen_dVb = dTcen_dVg * dVgC_dVb;
        dTcen_dVg *= dVgC_dVg;

        Ccen = epssub / Tcen;
        T0 = Cox / (Cox + Ccen);
        Coxeff = T0 * Ccen;
        T1 = -Ccen / Tcen;
        dCoxeff_dVg = T0 * T0 * T1;
        const double dCoxeff_dVd = dCoxeff_dVg * dTcen_dVd;
        dCoxeff_dVb = dCoxeff_dVg * dTcen_dVb;
        dCoxeff_dVg *= dTcen_dVg;
        CoxWLcen = CoxWL * Coxeff / coxe;

        const double AbulkCV = Abulk0 * P[kB4AbulkCVfactor];
        const double dAbulkCV_dVb = P[kB4AbulkCVfactor] * dAbulk0_dVb;
        const double VdsatCV = VgDP / AbulkCV;

        T0 = VdsatCV - Vds - kB4Delta4;
        const double dT0v_dVg = dVgDP_dVg / AbulkCV;
        const double dT0v_dVb = -VdsatCV * dAbulkCV_dVb / AbulkCV;
        T1 = sqrt(T0 * T0 + 4.0 * kB4Delta4 * VdsatCV);
        double dT1_dVg = (T0 + kB4Delta4 + kB4Delta4) / T1;
        const double dT1_dVd = -T0 / T1;
        const double dT1_dVb = dT1_dVg * dT0v_dVb;
        dT1_dVg *= dT0v_dVg;
        double VdseffCV, dVdseffCV_dVg, dVdseffCV_dVd, dVdseffCV_dVb;
        if (T0 >= 0.0) {
            VdseffCV = VdsatCV - 0.5 * (T0 + T1);
            dVdseffCV_dVg = 0.5 * (dT0v_dVg - dT1_dVg);
            dVdseffCV_dVd = 0.5 * (1.0 - dT1_dVd);
            dVdseffCV_dVb = 0.5 * (dT0v_dVb - dT1_dVb);
        } else {
            T3 = (kB4Delta4 + kB4Delta4) / (T1 - T0);
            const double T4 = 1.0 - T3;
            const double T5 = VdsatCV * T3 / (T1 - T0);
            VdseffCV = VdsatCV * T4;
            dVdseffCV_dVg = dT0v_dVg * T4 + T5 * (dT1_dVg - dT0v_dVg);
            dVdseffCV_dVd = T5 * (dT1_dVd + 1.0);
            dVdseffCV_dVb = dT0v_dVb * (T4 - T5) + T5 * dT1_dVb;
        }
        if (Vds == 0.0) {
            VdseffCV = 0.0;
            dVdseffCV_dVg = 0.0;
            dVdseffCV_dVb = 0.0;
        }

        T0 = AbulkCV * VdseffCV;
        T1 = VgDP;
        T2 = 12.0 * (T1 - 0.5 * T0 + 1.0e-20);
        T3 = T0 / T2;
        double T4 = 1.0 - 12.0 * T3 * T3;
        double T5 = AbulkCV * (6.0 * T0 * (4.0 * T1 - T0) / (T2 * T2) - 0.5);
        double T6 = T5 * VdseffCV / AbulkCV;

        qgate = CoxWLcen * (T1 - T0 * (0.5 - T3));
        QovCox = qgate / Coxeff;
        double Cgg1 = CoxWLcen * (T4 * dVgDP_dVg + T5 * dVdseffCV_dVg);
        const double Cgd1 = CoxWLcen * T5 * dVdseffCV_dVd + Cgg1 * dVgC_dVd + QovCox * dCoxeff_dVd;
        const double Cgb1 = CoxWLcen * (T5 * dVdseffCV_dVb + T6 * dAbulkCV_dVb) + Cgg1 * dVgC_dVb +
                            QovCox * dCoxeff_dVb;
        Cgg1 = Cgg1 * dVgC_dVg + QovCox * dCoxeff_dVg;

        double T7 = 1.0 - AbulkCV;
        double T8 = T2 * T2;
        const double T9 = 12.0 * T7 * T0 * T0 / (T8 * AbulkCV);
        const double T10 = T9 * dVgDP_dVg;
        const double T11 = -T7 * T5 / AbulkCV;
        const double T12 = -(T9 * T1 / AbulkCV + VdseffCV * (0.5 - T0 / T2));

        qbulk = CoxWLcen * T7 * (0.5 * VdseffCV - T0 * VdseffCV / T2);
        QovCox = qbulk / Coxeff;
        double Cbg1 = CoxWLcen * (T10 + T11 * dVdseffCV_dVg);
        const double Cbd1 = CoxWLcen * T11 * dVdseffCV_dVd + Cbg1 * dVgC_dVd + QovCox * dCoxeff_dVd;
        const double Cbb1 = CoxWLcen * (T11 * dVdseffCV_dVb + T12 * dAbulkCV_dVb) + Cbg1 * dVgC_dVb +
                            QovCox * dCoxeff_dVb;
        Cbg1 = Cbg1 * dVgC_dVg + QovCox * dCoxeff_dVg;

        double Csg, Csd, Csb;
        if (P[kB4Xpart] > 0.5) {  // 0/100 partition
            qsrc = -CoxWLcen * (T1 / 2.0 + T0 / 4.0 - 0.5 * T0 * T0 / T2);
            QovCox = qsrc / Coxeff;
            T2 += T2;
            T3 = T2 * T2;
            T7 = -(0.25 - 12.0 * T0 * (4.0 * T1 - T0) / T3);
            T4 = -(0.5 + 24.0 * T0 * T0 / T3) * dVgDP_dVg;
            T5 = T7 * AbulkCV;
            T6 = T7 * VdseffCV;
            Csg = CoxWLcen * (T4 + T5 * dVdseffCV_dVg);
            Csd = CoxWLcen * T5 * dVdseffCV_dVd + Csg * dVgC_dVd + QovCox * dCoxeff_dVd;
            Csb = CoxWLcen * (T5 * dVdseffCV_dVb + T6 * dAbulkCV_dVb) + Csg * dVgC_dVb +
                  QovCox * dCoxeff_dVb;
            Csg = Csg * dVgC_dVg + QovCox * dCoxeff_dVg;
        } else if (P[kB4Xpart] < 0.5) {  // 40/60 partition
            T2 = T2 / 12.0;
            T3 = 0.5 * CoxWLcen / (T2 * T2);
            T4 = T1 * (2.0 * T0 * T0 / 3.0 + T1 * (T1 - 4.0 * T0 / 3.0)) - 2.0 * T0 * T0 * T0 / 15.0;
            qsrc = -T3 * T4;
            QovCox = qsrc / Coxeff;
            T8 = 4.0 / 3.0 * T1 * (T1 - T0) + 0.4 * T0 * T0;
            T5 = -2.0 * qsrc / T2 - T3 * (T1 * (3.0 * T1 - 8.0 * T0 / 3.0) + 2.0 * T0 * T0 / 3.0);
            T6 = AbulkCV * (qsrc / T2 + T3 * T8);
            T7 = T6 * VdseffCV / AbulkCV;
            Csg = T5 * dVgDP_dVg + T6 * dVdseffCV_dVg;
            Csd = Csg * dVgC_dVd + T6 * dVdseffCV_dVd + QovCox * dCoxeff_dVd;
            Csb = Csg * dVgC_dVb + T6 * dVdseffCV_dVb + T7 * dAbulkCV_dVb + QovCox * dCoxeff_dVb;
            Csg = Csg * dVgC_dVg + QovCox * dCoxeff_dVg;
        } else {  // 50/50 partition
            qsrc = -0.5 * qgate;
            Csg = -0.5 * Cgg1;
            Csd = -0.5 * Cgd1;
            Csb = -0.5 * Cgb1;
        }
        qgate += Qac0 + Qsub0 - qbulk;
        qbulk -= (Qac0 + Qsub0);
        qdrn = -(qgate + qbulk + qsrc);

        const double Cbg = Cbg1 - dQac0_dVg - dQsub0_dVg;
        const double Cbd = Cbd1 - dQsub0_dVd;
        double Cbb = Cbb1 - dQac0_dVb - dQsub0_dVb;
        const double Cgg = Cgg1 - Cbg;
        const double Cgd = Cgd1 - Cbd;
        double Cgb = Cgb1 - Cbb;
        Cgb *= dVbseff_dVb;
        Cbb *= dVbseff_dVb;
        Csb *= dVbseff_dVb;

        cggb = Cgg;
        cgsb = -(Cgg + Cgd + Cgb);
        cgdb = Cgd;
        cdgb = -(Cgg + Cbg + Csg);
        cdsb = (Cgg + Cgd + Cgb + Cbg + Cbd + Cbb + Csg + Csd + Csb);
        cddb = -(Cgd + Cbd + Csd);
        cbgb = Cbg;
        cbsb = -(Cbg + Cbd + Cbb);
        cbdb = Cbd;
    }
    qsrc = -(qgate + qbulk + qdrn);

    // --- junction C-V (:3844-3950) ---
    double capbs = 0.0, capbd = 0.0;
    if (charge) {
        if (vbs_jct == 0.0) {
            s0[kB4SQbs] = 0.0;
            capbs = P[kB4Czbs] + P[kB4Czbssw] + P[kB4Czbsswg];
        } else if (vbs_jct < 0.0) {
            b4_junction_reverse(vbs_jct, P[kB4Czbs], P[kB4Czbssw], P[kB4Czbsswg], P[kB4PhiBS],
                                P[kB4PhiBSWS], P[kB4PhiBSWGS], P[kB4MJS], P[kB4MJSWS],
                                P[kB4MJSWGS], &s0[kB4SQbs], &capbs);
        } else {
            const double T0 = P[kB4Czbs] + P[kB4Czbssw] + P[kB4Czbsswg];
            const double T1 = vbs_jct * (P[kB4Czbs] * P[kB4MJS] / P[kB4PhiBS] +
                                         P[kB4Czbssw] * P[kB4MJSWS] / P[kB4PhiBSWS] +
                                         P[kB4Czbsswg] * P[kB4MJSWGS] / P[kB4PhiBSWGS]);
            s0[kB4SQbs] = vbs_jct * (T0 + 0.5 * T1);
            capbs = T0 + T1;
        }
        if (vbd_jct == 0.0) {
            s0[kB4SQbd] = 0.0;
            capbd = P[kB4Czbd] + P[kB4Czbdsw] + P[kB4Czbdswg];
        } else if (vbd_jct < 0.0) {
            b4_junction_reverse(vbd_jct, P[kB4Czbd], P[kB4Czbdsw], P[kB4Czbdswg], P[kB4PhiBD],
                                P[kB4PhiBSWD], P[kB4PhiBSWGD], P[kB4MJD], P[kB4MJSWD],
                                P[kB4MJSWGD], &s0[kB4SQbd], &capbd);
        } else {
            const double T0 = P[kB4Czbd] + P[kB4Czbdsw] + P[kB4Czbdswg];
            const double T1 = vbd_jct * (P[kB4Czbd] * P[kB4MJD] / P[kB4PhiBD] +
                                         P[kB4Czbdsw] * P[kB4MJSWD] / P[kB4PhiBSWD] +
                                         P[kB4Czbdswg] * P[kB4MJSWGD] / P[kB4PhiBSWGD]);
            s0[kB4SQbd] = vbd_jct * (T0 + 0.5 * T1);
            capbd = T0 + T1;
        }
    }

    // --- convergence test (:3952-4000) ---
    int noncon = 0;
    if (!off || !(mode & kM1InitFix)) {
        if (Check == 1) {
            noncon = 1;
        } else {
            const double Idn = (dmode >= 0) ? cdrain - cbd : cdrain + cbd;
            const double tol0 = reltol * m1_max(fabs(cdhat), fabs(Idn)) + abstol;
            if (fabs(cdhat - Idn) >= tol0) {
                noncon = 1;
            } else {
                const double Ibn = cbs + cbd;
                const double tol6 = reltol * m1_max(fabs(cbhat), fabs(Ibn)) + abstol;
                if (fabs(cbhat - Ibn) > tol6) noncon = 1;
            }
        }
    }
    (void)Idtot;
    (void)Ibtot;
    s0[kB4SVds] = vds;
    s0[kB4SVgs] = vgs;
    s0[kB4SVbs] = vbs;
    s0[kB4SVbd] = vbd;
    s0[kB4SVges] = vges;
    s0[kB4SVgms] = vgms;
    s0[kB4SVdbs] = vdbs;
    s0[kB4SVdbd] = vdbd;
    s0[kB4SVsbs] = vsbs;
    s0[kB4SVses] = vses;
    s0[kB4SVdes] = vdes;
    s0[kB4SQdef] = 0.0;

    // --- capacitance companion and charge integration (:4026-4546) ---
    double gcggb = 0, gcgdb = 0, gcgsb = 0, gcgbb = 0, gcdgb = 0, gcddb = 0, gcdsb = 0, gcdbb = 0;
    double gcsgb = 0, gcsdb = 0, gcssb = 0, gcsbb = 0, gcbdb = 0, gcbgb = 0, gcbsb = 0, gcbbb = 0;
    double ceqqg = 0.0, ceqqb = 0.0, ceqqd = 0.0;
    double sxpart, dxpart;
    if (charge) {
        double cgdo, qgdo, cgso, qgso;
        b4_overlap(vgd, P[kB4Cgdo], P[kB4WeffCV], P[kB4Cgdl], P[kB4Ckappad], &cgdo, &qgdo);
        b4_overlap(vgs, P[kB4Cgso], P[kB4WeffCV], P[kB4Cgsl], P[kB4Ckappas], &cgso, &qgso);
        const double ag0 = ic.ag0;
        const double cgbo = P[kB4Cgbo];
        if (dmode > 0) {
            qdrn -= qgdo;
            gcggb = (cggb + cgdo + cgso + cgbo) * ag0;
            gcgdb = (cgdb - cgdo) * ag0;
            gcgsb = (cgsb - cgso) * ag0;
            gcgbb = -(gcggb + gcgdb + gcgsb);
            gcdgb = (cdgb - cgdo) * ag0;
            gcsgb = -(cggb + cbgb + cdgb + cgso) * ag0;
            gcbgb = (cbgb - cgbo) * ag0;
            const double qgb = cgbo * vgb;
            qgate += qgdo + qgso + qgb;
            qbulk -= qgb;
            qsrc = -(qgate + qbulk + qdrn);
            gcddb = (cddb + capbd + cgdo) * ag0;
            gcdsb = cdsb * ag0;
            gcsdb = -(cgdb + cbdb + cddb) * ag0;
            gcssb = (capbs + cgso - (cgsb + cbsb + cdsb)) * ag0;
            gcdbb = -(gcdgb + gcddb + gcdsb + 0.0);
            gcsbb = -(gcsgb + gcsdb + gcssb + 0.0);
            gcbdb = (cbdb - capbd) * ag0;
            gcbsb = (cbsb - capbs) * ag0;
            gcbbb = -(gcbdb + gcbgb + gcbsb + 0.0);
            sxpart = 0.6;
            dxpart = 0.4;
        } else {
            qsrc = qdrn - qgso;
            gcggb = (cggb + cgdo + cgso + cgbo) * ag0;
            gcgdb = (cgsb - cgdo) * ag0;
            gcgsb = (cgdb - cgso) * ag0;
            gcgbb = -(gcggb + gcgdb + gcgsb);
            gcdgb = -(cggb + cbgb + cdgb + cgdo) * ag0;
            gcsgb = (cdgb - cgso) * ag0;
            gcbgb = (cbgb - cgbo) * ag0;
            const double qgb = cgbo * vgb;
            qgate += qgdo + qgso + qgb;
            qbulk -= qgb;
            qdrn = -(qgate + qbulk + qsrc);
            gcddb = (capbd + cgdo - (cgsb + cbsb + cdsb)) * ag0;
            gcdsb = -(cgdb + cbdb + cddb) * ag0;
            gcsdb = cdsb * ag0;
            gcssb = (cddb + capbs + cgso) * ag0;
            gcdbb = -(gcdgb + gcddb + gcdsb + 0.0);
            gcsbb = -(gcsgb + gcsdb + gcssb + 0.0);
            gcbdb = (cbsb - capbd) * ag0;
            gcbsb = (cbdb - capbs) * ag0;
            gcbbb = -(gcbgb + gcbdb + gcbsb + 0.0);
            sxpart = 0.4;
            dxpart = 0.6;
        }
        s0[kB4SQg] = qgate;
        s0[kB4SQd] = qdrn - s0[kB4SQbd];
        s0[kB4SQs] = qsrc - s0[kB4SQbs];
        s0[kB4SQb] = qbulk + s0[kB4SQbd] + s0[kB4SQbs];
        if (mode & kM1InitTran) {
            s1[kB4SQb] = s0[kB4SQb];
            s1[kB4SQg] = s0[kB4SQg];
            s1[kB4SQd] = s0[kB4SQd];
        }
        double geq, ceq;
        m1_integrate(ic, s0, s1, s2, kB4SQb, 0.0, &geq, &ceq);
        m1_integrate(ic, s0, s1, s2, kB4SQg, 0.0, &geq, &ceq);
        m1_integrate(ic, s0, s1, s2, kB4SQd, 0.0, &geq, &ceq);
        // equivalent charge currents (line860)
        const double cqgate = s0[kB4SCqg];
        const double cqbody = s0[kB4SCqb];
        const double cqdrn = s0[kB4SCqd];
        ceqqg = cqgate - gcggb * vgb + gcgdb * vbd + gcgsb * vbs;
        ceqqd = cqdrn - gcdgb * vgb - 0.0 * vgb + (gcddb + 0.0) * vbd - 0.0 * vbd_jct + gcdsb * vbs;
        ceqqb = cqbody - gcbgb * vgb - 0.0 * vgb + gcbdb * vbd + gcbsb * vbs;
        if (mode & kM1InitTran) {
            s1[kB4SCqb] = s0[kB4SCqb];
            s1[kB4SCqg] = s0[kB4SCqg];
            s1[kB4SCqd] = s0[kB4SCqd];
        }
    } else {
        // line850: no charge computation
        dxpart = (dmode > 0) ? 0.4 : 0.6;
        sxpart = 1.0 - dxpart;
    }
    (void)sxpart;
    (void)dxpart;

    // --- load current vector (line900, :4643-4870) ---
    double Gmx, Gmbsx, FwdSum, RevSum, ceqdrn;
    const double ceqbd = type * (0.0 - 0.0 * vds - 0.0 * vgs - 0.0 * vbs);
    double ceqbs;
    double gbbdp, gbbsp, gbdpg, gbdpdp, gbdpb, gbdpsp, gbspg, gbspdp, gbspb, gbspsp;
    if (dmode >= 0) {
        Gmx = gm;
        Gmbsx = gmbs;
        FwdSum = Gmx + Gmbsx;
        RevSum = 0.0;
        ceqdrn = type * (cdrain - gds * vds - Gmx * vgs - Gmbsx * vbs);
        ceqbs = type * (0.0 + 0.0 * vds - 0.0 * vgd - 0.0 * vbd);
        gbbdp = -(0.0);
        gbbsp = 0.0 + 0.0 + 0.0;
        gbdpg = 0.0;
        gbdpdp = 0.0;
        gbdpb = 0.0;
        gbdpsp = -(gbdpg + gbdpdp + gbdpb);
        gbspg = gbspdp = gbspb = gbspsp = 0.0;
    } else {
        Gmx = -gm;
        Gmbsx = -gmbs;
        FwdSum = 0.0;
        RevSum = -(Gmx + Gmbsx);
        ceqdrn = -type * (cdrain + gds * vds + Gmx * vgd + Gmbsx * vbd);
        ceqbs = type * (0.0 + 0.0 + (0.0 + 0.0) * vds - (0.0 + 0.0) * vgd - (0.0 + 0.0) * vbd);
        gbbsp = -(0.0);
        gbbdp = 0.0 + 0.0 + 0.0;
        gbdpg = gbdpsp = gbdpb = gbdpdp = 0.0;
        gbspg = 0.0;
        gbspsp = 0.0;
        gbspb = 0.0;
        gbspdp = -(gbspg + gbspsp + gbspb);
    }
    double ceqjs, ceqjd;
    if (type > 0) {
        ceqjs = (cbs - gbs * vbs_jct);
        ceqjd = (cbd - gbd * vbd_jct);
    } else {
        ceqjs = -(cbs - gbs * vbs_jct);
        ceqjd = -(cbd - gbd * vbd_jct);
        ceqqg = -ceqqg;
        ceqqd = -ceqqd;
        ceqqb = -ceqqb;
    }
    const double ceqgdtot = 0.0, ceqgstot = 0.0, ceqgcrg = 0.0, ceqqgmid = 0.0;
    const double Idtoteq = 0.0, Igtoteq = 0.0, Ibtoteq = 0.0, Istoteq = 0.0;
    t[kB4TRhsDP] = (ceqjd - ceqbd + ceqgdtot - ceqdrn - ceqqd + Idtoteq);
    t[kB4TRhsGP] = -(ceqqg - ceqgcrg + Igtoteq);
    t[kB4TRhsBP] = (ceqbd + ceqbs - ceqjd - ceqjs - ceqqb + Ibtoteq);
    t[kB4TRhsSP] = (ceqdrn - ceqbs + ceqjs + ceqqg + ceqqb + ceqqd + ceqqgmid - ceqgstot + Istoteq);

    // --- matrix (:4916-5015), m = 1 ---
    const double gjbd = gbd, gjbs = gbs, gdpr = 0.0, gspr = 0.0;
    const double gdtot = 0.0, gdtotd = 0.0, gdtotg = 0.0, gdtots = 0.0, gdtotb = 0.0;
    const double gstot = 0.0, gstotd = 0.0, gstotg = 0.0, gstots = 0.0, gstotb = 0.0;
    const double ggtg = 0.0, ggtd = 0.0, ggts = 0.0, ggtb = 0.0, T1q = 0.0;
    const double gIg = 0.0;  // gIgtot*, gIdtot*, gIstot*, gIbtot*
    const double dx0 = 0.0;  // ddxpart_dV*, dsxpart_dV*
    const double gbgs = 0.0, gbbs = 0.0;
    t[kB4TGPgp] = (gcggb - ggtg + gIg);
    t[kB4TGPdp] = (gcgdb - ggtd + gIg);
    t[kB4TGPsp] = (gcgsb - ggts + gIg);
    t[kB4TGPbp] = (gcgbb - ggtb + gIg);
    t[kB4TDPdp] = (gdpr + gds + gbd + T1q * dx0 - gdtotd + RevSum + gcddb + gbdpdp + dxpart * ggtd - gIg);
    t[kB4TDPd] = -((gdpr + gdtot));
    t[kB4TDPgp] = (Gmx + gcdgb - gdtotg + gbdpg - gIg + dxpart * ggtg + T1q * dx0);
    t[kB4TDPsp] = -((gds + gdtots - dxpart * ggts + gIg - T1q * dx0 + FwdSum - gcdsb - gbdpsp));
    t[kB4TDPbp] = -((gjbd + gdtotb - Gmbsx - gcdbb - gbdpb + gIg - T1q * dx0 - dxpart * ggtb));
    t[kB4TDdp] = -((gdpr - gdtotd));
    t[kB4TDd] = (gdpr + gdtot);
    t[kB4TSPdp] = -((gds + gstotd + RevSum - gcsdb - gbspdp - T1q * dx0 - sxpart * ggtd + gIg));
    t[kB4TSPgp] = (gcsgb - Gmx - gstotg + gbspg + sxpart * ggtg + T1q * dx0 - gIg);
    t[kB4TSPsp] = (gspr + gds + gbs + T1q * dx0 - gstots + FwdSum + gcssb + gbspsp + sxpart * ggts - gIg);
    t[kB4TSPs] = -((gspr + gstot));
    t[kB4TSPbp] = -((gjbs + gstotb + Gmbsx - gcsbb - gbspb - sxpart * ggtb - T1q * dx0 + gIg));
    t[kB4TSsp] = -((gspr - gstots));
    t[kB4TSs] = (gspr + gstot);
    t[kB4TBPdp] = (gcbdb - gjbd + gbbdp - gIg);
    t[kB4TBPgp] = (gcbgb - gbgs - gIg);
    t[kB4TBPsp] = (gcbsb - gjbs + gbbsp - gIg);
    t[kB4TBPbp] = (gjbd + gjbs + gcbbb - gbbs - gIg);

    rec[kB4RVon] = von_new;
    rec[kB4RMode] = static_cast<double>(dmode);
    rec[kB4RCd] = cdrain;
    rec[kB4RCbs] = cbs;
    rec[kB4RCbd] = cbd;
    rec[kB4RGbs] = gbs;
    rec[kB4RGbd] = gbd;
    rec[kB4RGm] = gm;
    rec[kB4RGds] = gds;
    rec[kB4RGmbs] = gmbs;
    rec[kB4RVdsat] = Vdsat;
    rec[kB4RNoncon] = noncon;
}

}  // namespace nsg
