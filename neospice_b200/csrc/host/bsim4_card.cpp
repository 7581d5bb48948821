// BSIM4.7 (LEVEL=14) model cards: parameter defaulting (BSIM4v7setup,
// src/devices/bsim4v7/bsim4v7_setup.cpp) and the temperature / size
// preprocessing (BSIM4v7temp, src/devices/bsim4v7/bsim4v7_temp.cpp:60-2320)
// of one instance at the circuit temperature 300.15 K = TNOM, evaluated with
// the same operations and the host's libm, so every value of the parameter
// block equals the reference's.  Supported cards: the default card with
// TOXE, VTH0 and U0 optionally given (no binning parameters, so every
// size-dependent value is the model value; the charge-thickness capacitance
// model, dioMod 1, no resistance or body networks); instances with W, L and
// DELVTO, one finger, no drain/source areas, perimeters or squares.
#include "circuit.hpp"

#include "kernels/bsim4_model.cuh"

#include <cctype>
#include <cmath>
#include <stdexcept>
#include <string>

namespace nsg {

namespace {

// The constants of bsim4v7_setup.cpp / bsim4v7_temp.cpp.
constexpr double kEps0 = 8.85418e-12;
constexpr double kEpsSi = 1.03594e-10;
constexpr double kPi = 3.141592654;
constexpr double kChargeQ = 1.60219e-19;
constexpr double kKboQ = 8.617087e-5;
constexpr double kMinExpT = 1.713908431e-15;
constexpr double kMaxExpT = 5.834617425e14;
constexpr double kExpThresholdT = 34.0;
constexpr double kDeltaT = 1.0e-9;

struct B4Given {
    bool toxe = false, vth0 = false, u0 = false;
    double toxe_v = 0.0, vth0_v = 0.0, u0_v = 0.0;
};

B4Given parse(const Bsim4Card& in) {
    B4Given g;
    for (const auto& [key0, val] : in.params) {
        std::string k;
        for (char ch : key0) k.push_back(static_cast<char>(std::tolower(static_cast<unsigned char>(ch))));
        if (k == "toxe") {
            g.toxe = true;
            g.toxe_v = val;
        } else if (k == "vth0" || k == "vtho") {
            g.vth0 = true;
            g.vth0_v = val;
        } else if (k == "u0") {
            g.u0 = true;
            g.u0_v = val;
        } else if (k == "level" || k == "version") {
            // LEVEL=14 selects the model; the version string is 4.7 only.
        } else {
            throw std::invalid_argument("BSIM4v7 card: parameter '" + key0 +
                                        "' is not supported (default card with TOXE, VTH0, U0)");
        }
    }
    if (g.toxe && !(g.toxe_v > 0.0)) throw std::invalid_argument("BSIM4v7 card: TOXE must be > 0");
    return g;
}

// (exp(x) - 1)^2 based short-channel factor of the temperature code.
double theta_factor(double T0) {
    if (T0 < kExpThresholdT) {
        const double T1 = exp(T0);
        const double T2 = T1 - 1.0;
        const double T3 = T2 * T2;
        const double T4 = T3 + 2.0 * T1 * kMinExpT;
        return T1 / T4;
    }
    return 1.0 / (kMaxExpT - 2.0);
}

}  // namespace

std::vector<double> bsim4_param_block(const Bsim4Card& card, double W, double L, double delvto) {
    const B4Given giv = parse(card);
    if (!(W > 0.0) || !(L > 0.0)) throw std::invalid_argument("BSIM4v7: W and L must be > 0");
    const double type = card.type >= 0 ? 1.0 : -1.0;
    const bool nmos = type > 0;
    std::vector<double> P(kBsim4Params, 0.0);
    const double nf = 1.0;

    // ---- BSIM4v7setup defaults (the values the load path reads) ----
    const double toxe = giv.toxe ? giv.toxe_v : 30.0e-10;
    const double toxp = toxe;    // !toxpGiven: toxp = toxe (then toxe - dtox, dtox = 0)
    const double toxm = toxe;
    const double dtox = 0.0;
    const double epsrox = 3.9;
    const double cdsc = 2.4e-4, cdscb = 0.0, cdscd = 0.0, cit = 0.0, nfactor = 1.0;
    const double xj = .15e-6, vsat = 8.0e4, a0 = 1.0, ags = 0.0, a1 = 0.0, a2 = 1.0;
    const double keta = -0.047, nsub = 6.0e16, ndep = 1.7e17, nsd = 1.0e20, phin = 0.0;
    const double xt = 1.55e-7, kt1 = -0.11, kt1l = 0.0, kt2 = 0.022, k3 = 80.0, k3b = 0.0;
    const double w0 = 2.5e-6, lpe0 = 1.74e-7, lpeb = 0.0, dvt0 = 2.2, dvt1 = 0.53;
    const double dvt2 = -0.032, dvt0w = 0.0, dvt1w = 5.3e6, dvt2w = -0.032, drout = 0.56;
    const double dsub = drout;
    const double vth0_model = giv.vth0 ? giv.vth0_v : (nmos ? 0.7 : -0.7);
    const double ua = 1.0e-9, ub = 1.0e-19, uc = -0.0465e-9, ud = 0.0;
    const double u0_model = giv.u0 ? giv.u0_v : (nmos ? 0.067 : 0.025);
    const double up = 0.0, lp = 1.0e-8, ute = -1.5;
    const double voff = -0.08, minv = 0.0, voffl = 0.0, delta = 0.01;
    const double rdsw = 200.0, rdswmin = 0.0, prwg = 1.0, prwb = 0.0, prt = 0.0;
    const double eta0 = 0.08, etab = -0.07, pclm = 1.3, pdibl1 = 0.39, pdibl2 = 0.0086;
    const double pdiblb = 0.0, pscbe1 = 4.24e8, pscbe2 = 1.0e-5, wr = 1.0, dwg = 0.0, dwb = 0.0;
    const double b0 = 0.0, b1 = 0.0, cgsl = 0.0, cgdl = 0.0, ckappas = 0.6;
    const double ckappad = ckappas;
    const double cf = 2.0 * epsrox * kEps0 / kPi * log(1.0 + 0.4e-6 / toxe);
    const double clc = 0.1e-6, cle = 0.6;
    const double Lint = 0.0, Wint = 0.0, dlc = Lint, dwc = Wint;
    const double acde_model = 1.0, moin = 15.0, noff = 1.0, voffcv = 0.0, ados = 1.0, bdos = 1.0;
    const double xpart = 0.0, vbm = -3.0, vfb_model = -1.0;
    const double xl = 0.0, xw = 0.0, tnom = kTNominal;
    const double Js = 1.0E-4, Jssw = 0.0, Jsswg = 0.0;  // drain side equal
    const double pbs = 1.0, pbsws = 1.0, pbswgs = pbsws;
    const double cjs = 5.0E-4, cjsws = 5.0E-10, cjswgs = cjsws;
    const double mjs = 0.5, mjsws = 0.33, mjswgs = mjsws;
    const double njs = 1.0;
    (void)dtox;

    // ---- BSIM4v7temp, model part (:60-405) ----
    const double Temp = kTNominal;
    const double epssub = kEpsSi;
    const double coxe = epsrox * kEps0 / toxe;
    const double coxp = epsrox * kEps0 / toxp;
    const double cgdo_model = 0.6 * xj * coxe;  // !cgdoGiven, dlc not given
    const double cgso_model = 0.6 * xj * coxe;
    const double cgbo_model = 2.0 * dwc * coxe;
    const double Tnom = tnom;
    const double TRatio = Temp / Tnom;
    const double vcrit = kB4Vt0 * log(kB4Vt0 / (kRoot2 * 1.0e-14));
    const double factor1 = sqrt(epssub / (epsrox * kEps0) * toxe);
    const double Vtm0 = kKboQ * Tnom;
    const double Eg0 = 1.16 - 7.02e-4 * Tnom * Tnom / (Tnom + 1108.0);
    const double ni = 1.45e10 * (Tnom / 300.15) * sqrt(Tnom / 300.15) *
                      exp(21.5565981 - Eg0 / (2.0 * Vtm0));
    const double vtm = kKboQ * Temp;
    (void)Eg0;
    // Temp == Tnom: saturation-current densities unchanged; delTemp = 0.
    const double delTemp = Temp - tnom;
    const double JsT = Js, JsswT = Jssw, JsswgT = Jsswg;
    double T0 = 0.0 * delTemp;  // TCJ = 0
    const double cjsT = cjs * (1.0 + T0);
    T0 = 0.0 * delTemp;         // TCJSW = 0
    const double cjswsT = cjsws * (1.0 + T0);
    T0 = 0.0 * delTemp;         // TCJSWG = 0
    const double cjswgsT = cjswgs * (1.0 + T0);
    const double PhiBS = pbs - 0.0 * delTemp;
    const double PhiBSWS = pbsws - 0.0 * delTemp;
    const double PhiBSWGS = pbswgs - 0.0 * delTemp;

    // ---- size-dependent parameters (:430-1525) ----
    const double Lnew = L + xl;
    const double Wnew = W / nf + xw;
    double T1, T2, T3, T4, T5, T8, T9, tmp, tmp1, tmp2;
    T0 = pow(Lnew, 1.0);   // Lln
    T1 = pow(Wnew, 1.0);   // Lwn
    tmp1 = 0.0 / T0 + 0.0 / T1 + 0.0 / (T0 * T1);
    const double dl = Lint + tmp1;
    tmp2 = 0.0 / T0 + 0.0 / T1 + 0.0 / (T0 * T1);
    const double dlcp = dlc + tmp2;
    T2 = pow(Lnew, 1.0);   // Wln
    T3 = pow(Wnew, 1.0);   // Wwn
    tmp1 = 0.0 / T2 + 0.0 / T3 + 0.0 / (T2 * T3);
    const double dw = Wint + tmp1;
    tmp2 = 0.0 / T2 + 0.0 / T3 + 0.0 / (T2 * T3);
    const double dwcp = dwc + tmp2;
    const double dwj = dwcp;  // setup: dwj = dwc; temp: dwj + tmp2
    const double dwjp = dwj + tmp2;
    const double leff = Lnew - 2.0 * dl;
    const double weff = Wnew - 2.0 * dw;
    const double leffCV = Lnew - 2.0 * dlcp;
    const double weffCV = Wnew - 2.0 * dwcp;
    const double weffCJ = Wnew - 2.0 * dwjp;
    if (!(leff > 0.0) || !(weff > 0.0) || !(leffCV > 0.0) || !(weffCV > 0.0) || !(weffCJ > 0.0))
        throw std::invalid_argument("BSIM4v7: effective channel length or width <= 0");
    // With no binning parameters every binned value is the model value.
    const double abulkCVfactor = 1.0 + pow((clc / leffCV), cle);
    T0 = (TRatio - 1.0);
    const double PowWeffWr = pow(weffCJ * 1.0e6, wr) * nf;
    const double T10r = prt * T0;
    const double rds0 = (rdsw + T10r) * nf / PowWeffWr;
    const double rdswminp = (rdswmin + T10r) * nf / PowWeffWr;
    double u0 = u0_model;
    if (u0 > 1.0) u0 = u0 / 1.0e4;
    T5 = 1.0 - up * exp(-leff / lp);
    const double u0temp = u0 * T5 * pow(TRatio, ute);
    const double uap = ua + 1.0e-9 * T0;          // ua1
    const double ubp = ub + -1.0e-18 * T0;        // ub1
    const double ucp = uc + -0.056e-9 * T0;       // uc1
    const double udp = ud + 0.0 * T0;             // ud1
    const double vsattemp = vsat - 3.3e4 * T0;    // at
    const double voffp = voff * (1.0 + 0.0 * delTemp);
    const double nfactorp = nfactor + 0.0 * delTemp / Tnom;
    const double voffcvp = voffcv * (1.0 + 0.0 * delTemp);
    const double eta0p = eta0 + 0.0 * delTemp / Tnom;
    const double cgdo = (cgdo_model + cf) * weffCV;
    const double cgso = (cgso_model + cf) * weffCV;
    const double cgbo = cgbo_model * leffCV * nf;
    const double phi = Vtm0 * log(ndep / ni) + phin + 0.4;
    const double sqrtPhi = sqrt(phi);
    const double Xdep0 = sqrt(2.0 * epssub / (kChargeQ * ndep * 1.0e6)) * sqrtPhi;
    const double litl = sqrt(3.0 * 3.9 / epsrox * xj * toxe);
    const double vbi = Vtm0 * log(nsd * ndep / (ni * ni));
    const double cdep0 = sqrt(kChargeQ * epssub * ndep * 1.0e6 / 2.0 / phi);
    const double mstar = 0.5 + atan(minv) / kPi;
    const double voffcbn = voffp + voffl / leff;
    const double ldeb = sqrt(epssub * Vtm0 / (kChargeQ * ndep * 1.0e6)) / 3.0;
    const double acde = acde_model * pow((ndep / 2.0e16), -0.25);
    // k1 / k2 from the doping (K1 and K2 not given)
    double vbx = phi - 7.7348e-4 * ndep * xt * xt;
    if (vbx > 0.0) vbx = -vbx;
    const double gamma1 = 5.753e-12 * sqrt(ndep) / coxe;
    const double gamma2 = 5.753e-12 * sqrt(nsub) / coxe;
    T0 = gamma1 - gamma2;
    T1 = sqrt(phi - vbx) - sqrtPhi;
    T2 = sqrt(phi * (phi - vbm)) - phi;
    const double k2 = T0 * T1 / (2.0 * T2 + vbm);
    const double k1 = gamma2 - 2.0 * k2 * sqrt(phi - vbm);
    double vfb = vfb_model;
    if (giv.vth0)
        vfb = type * vth0_model - phi - k1 * sqrtPhi;
    else
        vfb = -1.0;
    double vth0p = vth0_model;
    if (!giv.vth0) vth0p = type * (vfb + phi + k1 * sqrtPhi);
    const double k1ox = k1 * toxe / toxm;
    tmp = sqrt(epssub / (epsrox * kEps0) * toxe * Xdep0);
    T0 = dsub * leff / tmp;
    const double theta0vb0 = theta_factor(T0);
    T0 = drout * leff / tmp;
    T5 = theta_factor(T0);
    const double thetaRout = pdibl1 * T5 + pdibl2;
    tmp = sqrt(Xdep0);
    tmp1 = vbi - phi;
    tmp2 = factor1 * tmp;
    T0 = dvt1w * weff * leff / tmp2;
    T8 = theta_factor(T0);
    T0 = dvt0w * T8;
    T8 = T0 * tmp1;
    T0 = dvt1 * leff / tmp2;
    T9 = theta_factor(T0);
    T9 = dvt0 * T9 * tmp1;
    T4 = toxe * phi / (weff + w0);
    T0 = sqrt(1.0 + lpe0 / leff);
    T3 = (kt1 + kt1l / leff) * (TRatio - 1.0);
    T5 = k1ox * (T0 - 1.0) * sqrtPhi + T3;
    const double vfbzbfactor = -T8 - T9 + k3 * T4 + T5 - phi - k1 * sqrtPhi;
    (void)kDeltaT;

    // ---- instance part (:1560-2300), no stress or well-proximity effect ----
    double vth0 = vth0p;
    double k2i = k2;
    vth0 += delvto;
    vfb = vfb + type * delvto;
    T3 = type * vth0 - vfb - phi;
    T4 = T3 + T3;
    T5 = 2.5 * T3;
    double vtfbphi1 = nmos ? T4 : T5;
    if (vtfbphi1 < 0.0) vtfbphi1 = 0.0;
    double vtfbphi2 = 4.0 * T3;
    if (vtfbphi2 < 0.0) vtfbphi2 = 0.0;
    (void)vtfbphi1;
    double vbsc;
    if (k2i < 0.0) {
        T0 = 0.5 * k1 / k2i;
        vbsc = 0.9 * (phi - T0 * T0);
        if (vbsc > -3.0)
            vbsc = -3.0;
        else if (vbsc < -30.0)
            vbsc = -30.0;
    } else {
        vbsc = -30.0;
    }
    if (vbsc > vbm) vbsc = vbm;
    const double k2ox = k2i * toxe / toxm;
    const double vfbzb = vfbzbfactor + type * vth0;
    // BSIM4v7PAeffGeo, geoMod 0, one finger, DMCG = DMCI = DMDG = 0
    const double Pseff = 1.0 * ((0.0 + 0.0) + (0.0 + 0.0) + weffCJ) + 0.0 * (0.0 + 0.0);
    const double Pdeff = Pseff;
    const double Aseff = 1.0 * ((0.0 + 0.0) * weffCJ) + 0.0 * (0.0 * weffCJ);
    const double Adeff = Aseff;
    double SatCurS = 0.0, SatCurD = 0.0;
    if (!((Aseff <= 0.0) && (Pseff <= 0.0)))
        SatCurS = Aseff * JsT + Pseff * JsswT + weffCJ * nf * JsswgT;
    if (!((Adeff <= 0.0) && (Pdeff <= 0.0)))
        SatCurD = Adeff * JsT + Pdeff * JsswT + weffCJ * nf * JsswgT;
    if (SatCurS > 0.0 || SatCurD > 0.0)
        throw std::invalid_argument("BSIM4v7: junction saturation currents are not supported");

    // ---- the block ----
    P[kB4W] = W;
    P[kB4L] = L;
    P[kB4Delvto] = delvto;
    P[kB4Toxe] = toxe;
    P[kB4Type] = type;
    P[kB4IcVds] = P[kB4IcVgs] = P[kB4IcVbs] = 0.0;
    P[kB4Off] = 0.0;
    P[kB4Vtm] = vtm;
    P[kB4Vtm0] = Vtm0;
    P[kB4TempRatio] = Temp / tnom - 1.0;
    P[kB4Coxe] = coxe;
    P[kB4Coxp] = coxp;
    P[kB4Toxp] = toxp;
    P[kB4Factor1] = factor1;
    P[kB4Vcrit] = vcrit;
    P[kB4Ados] = ados;
    P[kB4Bdos] = bdos;
    P[kB4Xpart] = xpart;
    P[kB4Leff] = leff;
    P[kB4Weff] = weff;
    P[kB4LeffCV] = leffCV;
    P[kB4WeffCV] = weffCV;
    P[kB4WeffCJ] = weffCJ;
    P[kB4Phi] = phi;
    P[kB4SqrtPhi] = sqrtPhi;
    P[kB4Xdep0] = Xdep0;
    P[kB4Vbi] = vbi;
    P[kB4Dvt0] = dvt0;
    P[kB4Dvt1] = dvt1;
    P[kB4Dvt2] = dvt2;
    P[kB4Dvt0w] = dvt0w;
    P[kB4Dvt1w] = dvt1w;
    P[kB4Dvt2w] = dvt2w;
    P[kB4Lpe0] = lpe0;
    P[kB4Lpeb] = lpeb;
    P[kB4K1] = k1;
    P[kB4K1ox] = k1ox;
    P[kB4K3] = k3;
    P[kB4K3b] = k3b;
    P[kB4Kt1] = kt1;
    P[kB4Kt1l] = kt1l;
    P[kB4Kt2] = kt2;
    P[kB4W0] = w0;
    P[kB4Etab] = etab;
    P[kB4Theta0vb0] = theta0vb0;
    P[kB4Cit] = cit;
    P[kB4Nfactor] = nfactorp;
    P[kB4Cdsc] = cdsc;
    P[kB4Cdscb] = cdscb;
    P[kB4Cdscd] = cdscd;
    P[kB4Mstar] = mstar;
    P[kB4Voffcbn] = voffcbn;
    P[kB4Cdep0] = cdep0;
    P[kB4Dwg] = dwg;
    P[kB4Dwb] = dwb;
    P[kB4Prwg] = prwg;
    P[kB4Prwb] = prwb;
    P[kB4Rds0] = rds0;
    P[kB4Rdswmin] = rdswminp;
    P[kB4Xj] = xj;
    P[kB4A0] = a0;
    P[kB4Ags] = ags;
    P[kB4B0] = b0;
    P[kB4B1] = b1;
    P[kB4Keta] = keta;
    P[kB4Ua] = uap;
    P[kB4Ub] = ubp;
    P[kB4Uc] = ucp;
    P[kB4Ud] = udp;
    P[kB4A1] = a1;
    P[kB4A2] = a2;
    P[kB4Delta] = delta;
    P[kB4Pclm] = pclm;
    P[kB4Litl] = litl;
    P[kB4ThetaRout] = thetaRout;
    P[kB4Pdiblb] = pdiblb;
    P[kB4Pscbe1] = pscbe1;
    P[kB4Pscbe2] = pscbe2;
    P[kB4Vth0] = vth0;
    P[kB4K2ox] = k2ox;
    P[kB4Eta0] = eta0p;
    P[kB4U0temp] = u0temp;
    P[kB4Vsattemp] = vsattemp;
    P[kB4Vtfbphi2] = vtfbphi2;
    P[kB4Vbsc] = vbsc;
    P[kB4Vfbzb] = vfbzb;
    P[kB4Voffcv] = voffcvp;
    P[kB4Noff] = noff;
    P[kB4Acde] = acde;
    P[kB4Ldeb] = ldeb;
    P[kB4Moin] = moin;
    P[kB4AbulkCVfactor] = abulkCVfactor;
    P[kB4Cgdl] = cgdl;
    P[kB4Cgsl] = cgsl;
    P[kB4Ckappad] = ckappad;
    P[kB4Ckappas] = ckappas;
    P[kB4Cgdo] = cgdo;
    P[kB4Cgso] = cgso;
    P[kB4Cgbo] = cgbo;
    P[kB4SatCurS] = SatCurS;
    P[kB4SatCurD] = SatCurD;
    P[kB4NjS] = njs;
    P[kB4NjD] = njs;
    P[kB4VjsmFwd] = P[kB4IVjsmFwd] = P[kB4VjdmFwd] = P[kB4IVjdmFwd] = 0.0;
    P[kB4Czbs] = cjsT * Aseff;
    P[kB4Czbssw] = cjswsT * Pseff;
    P[kB4Czbsswg] = cjswgsT * weffCJ * nf;
    P[kB4Czbd] = cjsT * Adeff;
    P[kB4Czbdsw] = cjswsT * Pdeff;
    P[kB4Czbdswg] = cjswgsT * weffCJ * nf;
    P[kB4PhiBS] = PhiBS;
    P[kB4PhiBSWS] = PhiBSWS;
    P[kB4PhiBSWGS] = PhiBSWGS;
    P[kB4PhiBD] = PhiBS;
    P[kB4PhiBSWD] = PhiBSWS;
    P[kB4PhiBSWGD] = PhiBSWGS;
    P[kB4MJS] = mjs;
    P[kB4MJSWS] = mjsws;
    P[kB4MJSWGS] = mjswgs;
    P[kB4MJD] = mjs;
    P[kB4MJSWD] = mjsws;
    P[kB4MJSWGD] = mjswgs;
    return P;
}

}  // namespace nsg
