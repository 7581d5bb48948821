// Time-dependent independent-source values, shared by host and device:
// VSource/ISource::value_at for DC, PULSE and PWL
// (src/devices/vsource.cpp:80-131), operation for operation.
#pragma once
#include <cmath>

#ifdef __CUDACC__
#define NSG_HD __host__ __device__
#else
#define NSG_HD
#endif

namespace nsg {

// wave: 0 DC {v}, 1 PULSE {v1 v2 td tr tf pw per}, 2 PWL {t0 v0 t1 v1 ...}.
NSG_HD inline double wave_value(int wave, const double* p, int nparam, double t) {
    if (wave == 1) {
        const double v1 = p[0], v2 = p[1], td = p[2], tr = p[3], tf = p[4], pw = p[5], per = p[6];
        if (t < td) return v1;
        const double t_rel = t - td;
        const double t_in = (per > 0.0) ? fmod(t_rel, per) : t_rel;
        if (t_in < tr) return v1 + (v2 - v1) * (t_in / tr);
        if (t_in < tr + pw) return v2;
        if (t_in < tr + pw + tf) {
            const double t_fall = t_in - (tr + pw);
            return v2 + (v1 - v2) * (t_fall / tf);
        }
        return v1;
    }
    if (wave == 2) {
        const int npts = nparam / 2;
        if (npts == 0) return 0.0;
        if (t <= p[0]) return p[1];
        if (t >= p[2 * (npts - 1)]) return p[2 * (npts - 1) + 1];
        int hi = 1;
        for (; hi < npts; ++hi)
            if (p[2 * hi] >= t) break;
        const int lo = hi - 1;
        const double t0 = p[2 * lo], v0 = p[2 * lo + 1];
        const double t1 = p[2 * hi], v1 = p[2 * hi + 1];
        if (t1 == t0) return v1;
        const double frac = (t - t0) / (t1 - t0);
        return v0 + (v1 - v0) * frac;
    }
    return p[0];
}

}  // namespace nsg
