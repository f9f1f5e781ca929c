// Test infrastructure only: CPU restatement of MERCURY6's close-encounter
// record encoding, statement for statement: mio_ce's record body
// (mercury6_2.for:5456-5510), mio_fl2c (5885-5918), mio_re2c (6926-6957) and
// mco_x2ov (3057-3086). Fortran semantics kept: INT truncates toward zero,
// real MOD is fmod, 10.d0**(-ex) is gfortran's integer power (__builtin_powi),
// SIGN(y, x) takes x's sign, and the overlapping substring assignments of
// mio_ce leave each field the characters the next one does not overwrite.
#pragma once
#include <algorithm>
#include <cmath>

namespace oracle {

constexpr double IO_PI = 3.141592653589793;
constexpr double IO_TWOPI = IO_PI * 2.0;

// mio_re2c: x in [xmin, xmax) as 8 base-224 characters (32..255); 255s at or
// above xmax, blanks at or below xmin.
inline void mio_re2c(double x, double xmin, double xmax, unsigned char out[8]) {
    for (int j = 0; j < 8; ++j) out[j] = ' ';
    const double y = (x - xmin) / (xmax - xmin);
    if (y >= 1.0) {
        for (int j = 0; j < 8; ++j) out[j] = 255;
    } else if (y > 0.0) {
        double z = y;
        for (int j = 0; j < 8; ++j) {
            z = std::fmod(z, 1.0) * 224.0;
            out[j] = (unsigned char)((int)z + 32);
        }
    }
}

// mio_fl2c: 7 characters of mantissa and one of decimal exponent. The Fortran
// leaves the exponent undefined for x = 0; it is 0 here.
inline void mio_fl2c(double x, unsigned char out[8]) {
    int ex = 0;
    double y;
    if (x == 0.0) {
        y = 0.5;
    } else {
        const double ax = std::fabs(x);
        ex = (int)std::log10(ax);
        if (ax >= 1.0) ex = ex + 1;
        y = ax * __builtin_powi(10.0, -ex);
        if (y == 1.0) {
            y = y * 0.1;
            ex = ex + 1;
        }
        y = std::copysign(y, x) * 0.5 + 0.5;
    }
    mio_re2c(y, 0.0, 1.0, out);
    ex = ex + 112;
    if (ex > 223) ex = 223;
    if (ex < 0) ex = 0;
    out[7] = (unsigned char)(ex + 32);
}

// mco_x2ov with m = 0 (mio_ce's call): log-distance, angles, velocity ratio.
inline void mco_x2ov(double rcen, double rmax, double mcen, const double* xv, double& fr, double& theta,
                     double& phi, double& fv, double& vtheta, double& vphi) {
    const double x = xv[0], y = xv[1], z = xv[2], u = xv[3], v = xv[4], w = xv[5];
    const double r = std::sqrt(x * x + y * y + z * z);
    const double v2 = u * u + v * v + w * w;
    const double v1 = std::sqrt(v2);
    const double be = (mcen + 0.0) / r;
    const double ke = 0.5 * v2;
    fr = std::log10(std::min(std::max(r, rcen), rmax) / rcen);
    const double temp = ke / be;
    fv = 1.0 / (1.0 + 2.0 * temp * temp);
    theta = std::fmod(std::acos(z / r) + IO_TWOPI, IO_TWOPI);
    vtheta = std::fmod(std::acos(w / v1) + IO_TWOPI, IO_TWOPI);
    phi = std::fmod(std::atan2(y, x) + IO_TWOPI, IO_TWOPI);
    vphi = std::fmod(std::atan2(v, u) + IO_TWOPI, IO_TWOPI);
}

// mio_ce's record body c(1:70) for one close encounter (1-based ids i, j).
inline void mio_ce_record(double tclo, int i, int j, double dclo, const double* ixv, const double* jxv, double mcen,
                          double rcen, double rmax, unsigned char line[70]) {
    unsigned char c[80];
    for (int k = 0; k < 80; ++k) c[k] = ' ';
    auto put = [&](int first, int last, const unsigned char* s8) {  // c(first:last) = s8, 1-based
        for (int k = first; k <= last; ++k) c[k - 1] = k - first < 8 ? s8[k - first] : ' ';
    };
    unsigned char f[8];
    const double rfac = std::log10(rmax / rcen);
    mio_fl2c(tclo, f);
    put(1, 8, f);
    mio_re2c(double(i - 1), 0.0, 11239423.99, f);
    put(9, 16, f);
    mio_re2c(double(j - 1), 0.0, 11239423.99, f);
    put(12, 19, f);
    mio_fl2c(dclo, f);
    put(15, 22, f);
    const double* xv[2] = {ixv, jxv};
    const int base[2] = {23, 47};
    for (int b = 0; b < 2; ++b) {
        double fr, theta, phi, fv, vtheta, vphi;
        mco_x2ov(rcen, rmax, mcen, xv[b], fr, theta, phi, fv, vtheta, vphi);
        const int o = base[b];
        mio_re2c(fr, 0.0, rfac, f);
        put(o, o + 7, f);
        mio_re2c(theta, 0.0, IO_PI, f);
        put(o + 4, o + 11, f);
        mio_re2c(phi, 0.0, IO_TWOPI, f);
        put(o + 8, o + 15, f);
        mio_re2c(fv, 0.0, 1.0, f);
        put(o + 12, o + 19, f);
        mio_re2c(vtheta, 0.0, IO_PI, f);
        put(o + 16, b == 0 ? o + 23 : o + 27, f);
        mio_re2c(vphi, 0.0, IO_TWOPI, f);
        put(o + 20, b == 0 ? o + 27 : o + 31, f);
    }
    for (int k = 0; k < 70; ++k) line[k] = c[k];
}

}  // namespace oracle
