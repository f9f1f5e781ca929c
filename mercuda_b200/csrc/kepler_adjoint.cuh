// Adjoint of the Kepler drift: the transpose of the two-body state-transition
// matrix applied to a vector, for the exact flow that drift_one computes.
//
// With r0 = |x|, sigma0 = x.v, alpha = 2 mu / r0 - v.v and the universal
// anomaly s solving r0 G1(s) + sigma0 G2(s) + mu G3(s) = dt (G_k = s^k c_k(alpha
// s^2), c_k the Stumpff functions), the drift is x' = f x + g v, v' = fd x +
// gd v with f = 1 - mu G2/r0, g = r0 G1 + sigma0 G2, fd = -mu G1/(r r0),
// gd = 1 - mu G2/r, r = r0 G0 + sigma0 G1 + mu G2. f, g, fd, gd depend on the
// initial state only through (r0, sigma0, alpha), directly and through s
// (implicit: ds = -(dF)/r); with dG_k/ds = G_{k-1}, dG_0/ds = -alpha G1 and
// dG_k/dalpha = (k G_{k+2} - s G_{k+1}) / 2, the vector-Jacobian product
// needs only a handful of scalars. The flow's Jacobian does not depend on how
// drift_one reached its result (fast elliptic path, universal variables or
// ten substeps): the drift is the same map.
#pragma once
#include <math.h>

#ifdef __CUDACC__
#define MB200_HD __host__ __device__
#else
#define MB200_HD
#endif

namespace mb200 {

// Stumpff functions c0..c5 of z. For |z| < 1, c4 and c5 by their series and
// the rest by c_k = 1/k! - z c_{k+2}; beyond, the closed forms.
MB200_HD inline void stumpff6(double z, double c[6]) {
    if (fabs(z) < 1.0) {
        // c_k(z) = sum_j (-z)^j / (k + 2j)!, j = 0..11 (the next term is below
        // 1e-28 of the first), by Horner's rule on the coefficients 1/(k+2j)!
        const double C4[12] = {4.1666666666666664e-02, 1.388888888888889e-03,  2.48015873015873e-05,
                               2.755731922398589e-07,  2.08767569878681e-09,   1.1470745597729725e-11,
                               4.779477332387385e-14,  1.5619206968586225e-16, 4.110317623312165e-19,
                               8.896791392450574e-22,  1.6117375710961184e-24, 2.4795962632247976e-27};
        const double C5[12] = {8.333333333333333e-03,  1.984126984126984e-04,  2.7557319223985893e-06,
                               2.505210838544172e-08,  1.6059043836821613e-10, 7.647163731819816e-13,
                               2.8114572543455206e-15, 8.22063524662433e-18,   1.9572941063391263e-20,
                               3.868170170630684e-23,  6.446950284384474e-26,  9.183689863795546e-29};
        const double w = -z;
        double s4 = C4[11], s5 = C5[11];
#pragma unroll
        for (int j = 10; j >= 0; --j) {
            s4 = fma(s4, w, C4[j]);
            s5 = fma(s5, w, C5[j]);
        }
        c[4] = s4;
        c[5] = s5;
        c[2] = 0.5 - z * s4;
        c[3] = 1.0 / 6.0 - z * s5;
        c[0] = 1.0 - z * c[2];
        c[1] = 1.0 - z * c[3];
        return;
    }
    if (z > 0.0) {
        const double w = sqrt(z), sw = sin(w), cw = cos(w);
        c[0] = cw;
        c[1] = sw / w;
        c[2] = (1.0 - cw) / z;
        c[3] = (w - sw) / (z * w);
    } else {
        const double w = sqrt(-z), sw = sinh(w), cw = cosh(w);
        c[0] = cw;
        c[1] = sw / w;
        c[2] = (cw - 1.0) / (-z);
        c[3] = (sw - w) / (-z * w);
    }
    c[4] = (0.5 - c[2]) / z;
    c[5] = (1.0 / 6.0 - c[3]) / z;
}

// G_0..G_5 at (s, alpha).
MB200_HD inline void gfuncs(double s, double alpha, double G[6]) {
    double c[6];
    stumpff6(alpha * s * s, c);
    double p = 1.0;
    for (int k = 0; k < 6; ++k) {
        G[k] = p * c[k];
        p *= s;
    }
}

// A starting value of the universal anomaly from the drift's end position x1:
// g and f follow from x x x1 = g (x x v) and x1 x v = f (x x v), then
// G2 = (1 - f) r0 / mu, G1 = (g - sigma0 G2) / r0, G0 = 1 - alpha G2, and s is
// the angle (or hyperbolic angle) with cosine G0 and sine sqrt(alpha) G1.
MB200_HD inline double anomaly_guess(const double x[3], const double v[3], const double x1[3], double r0,
                                     double sig0, double alpha, double mu, double dt) {
    const double h[3] = {x[1] * v[2] - x[2] * v[1], x[2] * v[0] - x[0] * v[2], x[0] * v[1] - x[1] * v[0]};
    const double hh = h[0] * h[0] + h[1] * h[1] + h[2] * h[2];
    const double fallback = dt / r0;
    if (!(hh > 0.0)) return fallback;
    const double a[3] = {x[1] * x1[2] - x[2] * x1[1], x[2] * x1[0] - x[0] * x1[2], x[0] * x1[1] - x[1] * x1[0]};
    const double b[3] = {x1[1] * v[2] - x1[2] * v[1], x1[2] * v[0] - x1[0] * v[2], x1[0] * v[1] - x1[1] * v[0]};
    const double g = (a[0] * h[0] + a[1] * h[1] + a[2] * h[2]) / hh;
    const double f = (b[0] * h[0] + b[1] * h[1] + b[2] * h[2]) / hh;
    const double G2 = (1.0 - f) * r0 / mu;
    const double G1 = (g - sig0 * G2) / r0;
    double s;
    if (alpha > 0.0) {
        const double w = sqrt(alpha);
        s = atan2(w * G1, 1.0 - alpha * G2) / w;
    } else if (alpha < 0.0) {
        const double w = sqrt(-alpha);
        s = asinh(w * G1) / w;
    } else {
        s = G1;
    }
    return isfinite(s) ? s : fallback;
}

// The universal anomaly of a drift of dt (Laguerre iteration on the universal
// Kepler equation from s). Returns false if it did not converge.
MB200_HD inline bool universal_anomaly(double r0, double sig0, double alpha, double mu, double dt, double& s) {
    for (int it = 0; it < 60; ++it) {
        double G[6];
        gfuncs(s, alpha, G);
        const double F = r0 * G[1] + sig0 * G[2] + mu * G[3] - dt;
        const double F1 = r0 * G[0] + sig0 * G[1] + mu * G[2];
        const double F2 = sig0 * G[0] + (mu - alpha * r0) * G[1];
        const double n = 5.0;
        const double disc = fabs((n - 1.0) * (n - 1.0) * F1 * F1 - n * (n - 1.0) * F * F2);
        const double den = F1 + copysign(sqrt(disc), F1);
        const double ds = den != 0.0 ? n * F / den : 0.0;
        s -= ds;
        if (!isfinite(s)) return false;
        if (fabs(ds) <= 4e-15 * fabs(s)) return true;
    }
    // rounding may keep the last correction just above the bound: accept a
    // root whose residual is at the rounding level of the equation's terms
    double G[6];
    gfuncs(s, alpha, G);
    const double F = r0 * G[1] + sig0 * G[2] + mu * G[3] - dt;
    const double scale = fabs(r0 * G[1]) + fabs(sig0 * G[2]) + fabs(mu * G[3]) + fabs(dt);
    return fabs(F) <= 1e-13 * scale;
}

// lx = d(x')/dx ^T lx1 + d(v')/dx ^T lv1, lv likewise, for the drift of
// (x, v) by dt about mu that ended at x1. Returns false if the anomaly did not
// converge.
MB200_HD inline bool drift_vjp(double mu, const double x[3], const double v[3], double dt, const double x1[3],
                              const double lx1[3], const double lv1[3], double lx[3], double lv[3]) {
    const double r0 = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    const double sig0 = x[0] * v[0] + x[1] * v[1] + x[2] * v[2];
    const double vv = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    const double alpha = 2.0 * mu / r0 - vv;
    double s = anomaly_guess(x, v, x1, r0, sig0, alpha, mu, dt);
    if (!universal_anomaly(r0, sig0, alpha, mu, dt, s)) return false;
    double G[6];
    gfuncs(s, alpha, G);
    const double r = r0 * G[0] + sig0 * G[1] + mu * G[2];
    const double f = 1.0 - mu * G[2] / r0;
    const double g = r0 * G[1] + sig0 * G[2];
    const double fd = -mu * G[1] / (r * r0);
    const double gd = 1.0 - mu * G[2] / r;
    // derivatives of G0..G3 with respect to alpha (fixed s) and s
    double Ga[4], Gs[4];
    for (int k = 0; k < 4; ++k) Ga[k] = 0.5 * (k * G[k + 2] - s * G[k + 1]);
    Gs[0] = -alpha * G[1];
    for (int k = 1; k < 4; ++k) Gs[k] = G[k - 1];
    // ds/dtheta for theta = r0, sigma0, alpha
    const double Fa = r0 * Ga[1] + sig0 * Ga[2] + mu * Ga[3];
    const double dsd[3] = {-G[1] / r, -G[2] / r, -Fa / r};
    const double ra = r0 * Ga[0] + sig0 * Ga[1] + mu * Ga[2];
    const double rs = r0 * Gs[0] + sig0 * Gs[1] + mu * Gs[2];
    const double c1 = lx1[0] * x[0] + lx1[1] * x[1] + lx1[2] * x[2];
    const double c2 = lx1[0] * v[0] + lx1[1] * v[1] + lx1[2] * v[2];
    const double c3 = lv1[0] * x[0] + lv1[1] * x[1] + lv1[2] * x[2];
    const double c4 = lv1[0] * v[0] + lv1[1] * v[1] + lv1[2] * v[2];
    double DS[3];
    for (int t = 0; t < 3; ++t) {
        const double is_r0 = t == 0 ? 1.0 : 0.0, is_sig = t == 1 ? 1.0 : 0.0, is_a = t == 2 ? 1.0 : 0.0;
        double DG[4];
        for (int k = 0; k < 4; ++k) DG[k] = is_a * Ga[k] + Gs[k] * dsd[t];
        const double DR = is_r0 * G[0] + is_sig * G[1] + is_a * ra + rs * dsd[t];
        const double Df = -mu * DG[2] / r0 + is_r0 * mu * G[2] / (r0 * r0);
        const double Dg = is_r0 * G[1] + is_sig * G[2] + r0 * DG[1] + sig0 * DG[2];
        const double rr0 = r * r0;
        const double Dfd = -mu * (DG[1] / rr0 - G[1] * (DR * r0 + r * is_r0) / (rr0 * rr0));
        const double Dgd = -mu * (DG[2] / r - G[2] * DR / (r * r));
        DS[t] = c1 * Df + c2 * Dg + c3 * Dfd + c4 * Dgd;
    }
    const double kx = DS[0] / r0 - DS[2] * 2.0 * mu / (r0 * r0 * r0);
    for (int c = 0; c < 3; ++c) {
        lx[c] = f * lx1[c] + fd * lv1[c] + kx * x[c] + DS[1] * v[c];
        lv[c] = g * lx1[c] + gd * lv1[c] + DS[1] * x[c] - 2.0 * DS[2] * v[c];
    }
    return true;
}

}  // namespace mb200
