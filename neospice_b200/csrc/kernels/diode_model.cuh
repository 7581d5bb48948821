// DC load of the level-1 junction diode (RS = 0, no breakdown, no knee
// currents, T = TNOM), shared by the host (first-iteration values for the
// symbolic phase) and the GPU Newton kernel.  Follows DIOload
// (src/devices/dio/dio_load.cpp:98-383) and DEVpnjlim
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
    int check;  // 1: limited / junction-init iteration (counts as non-converged)
};

// csat = area-scaled saturation current at T, vte = N*vt, tvcrit = Vcrit.
NSG_HD inline DiodeDC diode_dc_load(bool initjct, double v_pos, double v_neg, double vd_old,
                                    double csat, double vte, double tvcrit, double gmin) {
    DiodeDC r;
    r.check = 1;
    double vd;
    if (initjct) {
        vd = tvcrit;
    } else {
        vd = v_pos - v_neg;
        vd = pnjlim(vd, vd_old, vte, tvcrit, &r.check);
    }
    double cd, gd;
    if (vd >= -3 * vte) {
        const double evd = exp(vd / vte);
        cd = csat * (evd - 1);
        gd = csat * evd / vte;
    } else {
        double arg = 3 * vte / (vd * 2.7182818284590452354);
        arg = arg * arg * arg;
        cd = -csat * (1 + arg);
        gd = csat * 3 * arg / vd;
    }
    cd = cd + 0.0;  // + sidewall current (absent)
    gd = gd + 0.0;
    gd = gd + gmin;
    cd = cd + gmin * vd;
    r.vd = vd;
    r.cd = cd;
    r.gd = gd;
    return r;
}

// Vcrit of DIOtemp (src/devices/dio/dio_temp.cpp:209-212).
NSG_HD inline double diode_vcrit(double vte, double csat) {
    return vte * log(vte / (1.4142135623730950488 * csat));
}

}  // namespace nsg
