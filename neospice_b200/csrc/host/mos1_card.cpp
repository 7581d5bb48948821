// Level-1 MOSFET model cards: parameter defaulting (MOS1setup,
// src/devices/mos1/mos1_setup.cpp:24-100) and temperature preprocessing
// (MOS1temp, src/devices/mos1/mos1_temp.cpp:21-340) at the circuit
// temperature (TNOM 300.15 K), evaluated with the same operations and the host's
// libm, so every constant equals the reference's bit for bit.
#include "circuit.hpp"

#include "kernels/mos1_model.cuh"

#include <cctype>
#include <cmath>
#include <stdexcept>
#include <string>

namespace nsg {

namespace {

constexpr double kBoltz = 1.38064852e-23;
constexpr double kCharge = 1.6021766208e-19;
constexpr double kRefTemp = 300.15;
constexpr double kCtoK = 273.15;

struct Given {
    bool on = false;
    double v = 0.0;
};

struct Card {
    Given vto, kp, gamma, phi, lambda, rd, rs, cbd, cbs, is, pb, cgso, cgdo, cgbo, rsh, cj, mj,
        cjsw, mjsw, js, tox, ld, u0, fc, nsub, tpg, nss, tnom;
};

Card parse(const Mos1Card& in) {
    Card c;
    for (const auto& [key0, val] : in.params) {
        std::string k;
        for (char ch : key0) k.push_back(static_cast<char>(std::tolower(static_cast<unsigned char>(ch))));
        Given* g = nullptr;
        if (k == "vto" || k == "vt0") g = &c.vto;
        else if (k == "kp") g = &c.kp;
        else if (k == "gamma") g = &c.gamma;
        else if (k == "phi") g = &c.phi;
        else if (k == "lambda") g = &c.lambda;
        else if (k == "rd") g = &c.rd;
        else if (k == "rs") g = &c.rs;
        else if (k == "cbd") g = &c.cbd;
        else if (k == "cbs") g = &c.cbs;
        else if (k == "is") g = &c.is;
        else if (k == "pb") g = &c.pb;
        else if (k == "cgso") g = &c.cgso;
        else if (k == "cgdo") g = &c.cgdo;
        else if (k == "cgbo") g = &c.cgbo;
        else if (k == "rsh") g = &c.rsh;
        else if (k == "cj") g = &c.cj;
        else if (k == "mj") g = &c.mj;
        else if (k == "cjsw") g = &c.cjsw;
        else if (k == "mjsw") g = &c.mjsw;
        else if (k == "js") g = &c.js;
        else if (k == "tox") g = &c.tox;
        else if (k == "ld") g = &c.ld;
        else if (k == "u0" || k == "uo") g = &c.u0;
        else if (k == "fc") g = &c.fc;
        else if (k == "nsub") g = &c.nsub;
        else if (k == "tpg") g = &c.tpg;
        else if (k == "nss") g = &c.nss;
        else if (k == "tnom") g = &c.tnom;
        else if (k == "kf" || k == "af" || k == "level") continue;  // noise / level: no effect here
        else throw std::invalid_argument("MOS1 model: unknown parameter '" + key0 + "'");
        g->on = true;
        g->v = (k == "tnom") ? val + kCtoK : val;  // MOS1mParam stores TNOM in kelvin
        if (k == "tpg") g->v = static_cast<double>(static_cast<int>(val));
    }
    // MOS1setup gives a terminal an internal node when RD (RS) or RSH is
    // nonzero, MOS1temp a conductance from RD (RS) when given, else from
    // RSH: they disagree only for RD = 0 (RS = 0) given beside RSH != 0 (a
    // node without conductance), which is refused.
    if (c.rsh.on && c.rsh.v != 0.0 && ((c.rd.on && c.rd.v == 0.0) || (c.rs.on && c.rs.v == 0.0)))
        throw std::invalid_argument("MOS1 model: RD = 0 or RS = 0 given with RSH != 0 is not "
                                    "supported");
    return c;
}

double val(const Given& g, double dflt) { return g.on ? g.v : dflt; }

}  // namespace

std::vector<double> mos1_param_block(const Mos1Card& in, double W, double L, double circuit_temp) {
    if (in.type != 1 && in.type != -1) throw std::invalid_argument("MOS1 model: type must be +1 or -1");
    const Card c = parse(in);
    const double type = in.type;
    // MOS1setup defaults
    const double latDiff = val(c.ld, 0);
    const double jsDens = val(c.js, 0);
    const double jsat = val(c.is, 1e-14);
    double kp = val(c.kp, 2e-5);
    const double cgso = val(c.cgso, 0), cgdo = val(c.cgdo, 0), cgbo = val(c.cgbo, 0);
    double vt0 = val(c.vto, 0);
    const double cj = val(c.cj, 0), cjsw = val(c.cjsw, 0);
    const double pb = val(c.pb, .8);
    const double mj = val(c.mj, .5), mjsw = val(c.mjsw, .5);
    const double fc = val(c.fc, .5);
    double phi = val(c.phi, .6);
    const double lambda = val(c.lambda, 0);
    double gamma = val(c.gamma, 0);

    // MOS1temp, model part
    const double tnom = val(c.tnom, 300.15);
    const double fact1 = tnom / kRefTemp;
    const double vtnom = tnom * kKoverQ;
    const double kt1 = kBoltz * tnom;
    const double egfet1 = 1.16 - (7.02e-4 * tnom * tnom) / (tnom + 1108);
    const double arg1 = -egfet1 / (kt1 + kt1) + 1.1150877 / (kBoltz * (kRefTemp + kRefTemp));
    const double pbfact1 = -2 * vtnom * (1.5 * std::log(fact1) + kCharge * arg1);
    if (phi <= 0.0) throw std::invalid_argument("MOS1 model: Phi is not positive");
    double oxideCapFactor = 0.0;
    if (c.tox.on && c.tox.v != 0) {
        oxideCapFactor = 3.9 * 8.854214871e-12 / c.tox.v;
        if (!c.kp.on) kp = val(c.u0, 600) * oxideCapFactor * 1e-4;
        if (c.nsub.on) {
            if (c.nsub.v * 1e6 > 1.45e16) {
                if (!c.phi.on) {
                    phi = 2 * vtnom * std::log(c.nsub.v * 1e6 / 1.45e16);
                    phi = (.1 > phi) ? .1 : phi;
                }
                const double fermis = type * .5 * phi;
                double wkfng = 3.2;
                const double tpg = val(c.tpg, 1);
                if (tpg != 0) {
                    const double fermig = type * tpg * .5 * egfet1;
                    wkfng = 3.25 + .5 * egfet1 - fermig;
                }
                const double wkfngs = wkfng - (3.25 + .5 * egfet1 + fermis);
                if (!c.gamma.on)
                    gamma = std::sqrt(2 * 11.70 * 8.854214871e-12 * kCharge * c.nsub.v * 1e6) /
                            oxideCapFactor;
                if (!c.vto.on) {
                    const double nss = val(c.nss, 0);
                    const double vfb = wkfngs - nss * 1e4 * kCharge / oxideCapFactor;
                    vt0 = vfb + type * (gamma * std::sqrt(phi) + phi);
                }
            } else {
                throw std::invalid_argument("MOS1 model: Nsub < Ni");
            }
        }
    }

    // MOS1temp, instance part (T = the circuit temperature, M = 1,
    // AD = AS = PD = PS = 0)
    if (!(circuit_temp > 0.0) || !std::isfinite(circuit_temp))
        throw std::invalid_argument("MOS1: temperature must be positive (kelvin)");
    const double temp = circuit_temp + 0.0;  // MOS1temp: CKTtemp + dtemp
    const double m = 1.0, drainArea = 0.0, sourceArea = 0.0, drainPerim = 0.0, sourcePerim = 0.0;
    const double vt = temp * kKoverQ;
    const double ratio = temp / tnom;
    const double fact2 = temp / kRefTemp;
    const double kt = temp * kBoltz;
    const double egfet = 1.16 - (7.02e-4 * temp * temp) / (temp + 1108);
    const double arg = -egfet / (kt + kt) + 1.1150877 / (kBoltz * (kRefTemp + kRefTemp));
    const double pbfact = -2 * vt * (1.5 * std::log(fact2) + kCharge * arg);
    const double ratio4 = ratio * std::sqrt(ratio);
    const double tTrans = kp / ratio4;
    const double phio = (phi - pbfact1) / fact1;
    const double tPhi = fact2 * phio + pbfact;
    const double tSatCur = jsat * std::exp(-egfet / vt + egfet1 / vtnom);
    const double tSatCurDens = jsDens * std::exp(-egfet / vt + egfet1 / vtnom);
    const double pbo = (pb - pbfact1) / fact1;
    const double gmaold = (pb - pbo) / pbo;
    double capfact = 1 / (1 + mj * (4e-4 * (tnom - kRefTemp) - gmaold));
    double tCbd = val(c.cbd, 0) * capfact;
    double tCbs = val(c.cbs, 0) * capfact;
    double tCj = cj * capfact;
    capfact = 1 / (1 + mjsw * (4e-4 * (tnom - kRefTemp) - gmaold));
    double tCjsw = cjsw * capfact;
    const double tBulkPot = fact2 * pbo + pbfact;
    const double gmanew = (tBulkPot - pbo) / pbo;
    capfact = (1 + mj * (4e-4 * (temp - kRefTemp) - gmanew));
    tCbd *= capfact;
    tCbs *= capfact;
    tCj *= capfact;
    capfact = (1 + mjsw * (4e-4 * (temp - kRefTemp) - gmanew));
    tCjsw *= capfact;
    const double tDepCap = fc * tBulkPot;
    double drainVcrit, sourceVcrit;
    if ((tSatCurDens == 0) || (drainArea == 0) || (sourceArea == 0)) {
        sourceVcrit = drainVcrit = vt * std::log(vt / (kRoot2 * m * tSatCur));
    } else {
        drainVcrit = vt * std::log(vt / (kRoot2 * m * tSatCurDens * drainArea));
        sourceVcrit = vt * std::log(vt / (kRoot2 * m * tSatCurDens * sourceArea));
    }
    auto junction = [&](bool capGiven, double tCap, double area, double perim, double* cz,
                        double* czsw, double* f2, double* f3, double* f4) {
        if (capGiven) *cz = tCap * m;
        else *cz = c.cj.on ? tCj * m * area : 0;
        *czsw = c.cjsw.on ? tCjsw * perim * m : 0;
        const double a = 1 - fc;
        const double sarg = std::exp((-mj) * std::log(a));
        const double sargsw = std::exp((-mjsw) * std::log(a));
        *f2 = *cz * (1 - fc * (1 + mj)) * sarg / a + *czsw * (1 - fc * (1 + mjsw)) * sargsw / a;
        *f3 = *cz * mj * sarg / a / tBulkPot + *czsw * mjsw * sargsw / a / tBulkPot;
        *f4 = *cz * tBulkPot * (1 - a * sarg) / (1 - mj) +
              *czsw * tBulkPot * (1 - a * sargsw) / (1 - mjsw) - *f3 / 2 * (tDepCap * tDepCap) -
              tDepCap * *f2;
    };
    double czbd, czbdsw, f2d, f3d, f4d, czbs, czbssw, f2s, f3s, f4s;
    junction(c.cbd.on, tCbd, drainArea, drainPerim, &czbd, &czbdsw, &f2d, &f3d, &f4d);
    junction(c.cbs.on, tCbs, sourceArea, sourcePerim, &czbs, &czbssw, &f2s, &f3s, &f4s);

    std::vector<double> P(kMos1Params, 0.0);
    P[kMW] = W;
    P[kML] = L;
    P[kMVto] = vt0;
    P[kMType] = type;
    P[kMM] = m;
    P[kMLatDiff] = latDiff;
    P[kMLambda] = lambda;
    P[kMGamma] = gamma;
    P[kMPhi] = phi;
    P[kMTPhi] = tPhi;
    P[kMEgHalfDiff] = .5 * (egfet1 - egfet);
    P[kMTTrans] = tTrans;
    P[kMTSatCur] = tSatCur;
    P[kMTSatCurDens] = tSatCurDens;
    P[kMDrainArea] = drainArea;
    P[kMSourceArea] = sourceArea;
    P[kMOxCapFactor] = oxideCapFactor;
    P[kMCgso] = cgso;
    P[kMCgdo] = cgdo;
    P[kMCgbo] = cgbo;
    P[kMSourceVcrit] = sourceVcrit;
    P[kMDrainVcrit] = drainVcrit;
    P[kMTBulkPot] = tBulkPot;
    P[kMTDepCap] = tDepCap;
    P[kMCbd] = czbd;
    P[kMCbdsw] = czbdsw;
    P[kMCbs] = czbs;
    P[kMCbssw] = czbssw;
    P[kMF2d] = f2d;
    P[kMF3d] = f3d;
    P[kMF4d] = f4d;
    P[kMF2s] = f2s;
    P[kMF3s] = f3s;
    P[kMF4s] = f4s;
    P[kMMj] = mj;
    P[kMMjsw] = mjsw;
    P[kMVt] = kKoverQ * temp;
    // MOS1temp's series conductances (mos1_temp.cpp:298-334): M / RD (M / RS)
    // when given, else M / (RSH * NRD) (NRS) with the default one square.
    const double drainSquares = 1, sourceSquares = 1;
    if (c.rd.on) {
        if (c.rd.v != 0) P[kMDrainCond] = m / c.rd.v;
    } else if (c.rsh.on) {
        if (c.rsh.v != 0) P[kMDrainCond] = m / (c.rsh.v * drainSquares);
    }
    if (c.rs.on) {
        if (c.rs.v != 0) P[kMSourceCond] = m / c.rs.v;
    } else if (c.rsh.on) {
        if ((c.rsh.v != 0) && (sourceSquares != 0))
            P[kMSourceCond] = m / (c.rsh.v * sourceSquares);
    }
    return P;  // initial conditions and OFF stay 0
}

}  // namespace nsg
