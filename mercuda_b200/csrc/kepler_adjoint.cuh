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

// Stumpff functions c0..c5 of z: closed forms for |z| >= 1, series below.
MB200_HD inline void stumpff6(double z, double c[6]) {
    if (fabs(z) < 1.0) {
        // c_k(z) = sum_j (-z)^j / (k + 2j)!
        for (int k = 0; k < 6; ++k) {
            double fact = 1.0;
            for (int q = 2; q <= k; ++q) fact *= q;
            double term = 1.0 / fact, sum = term;
            for (int j = 1; j < 14; ++j) {
                term = term * (-z) / ((double)(k + 2 * j - 1) * (double)(k + 2 * j));
                sum += term;
            }
            c[k] = sum;
        }
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

// The universal anomaly of a drift of dt (Laguerre iteration on the universal
// Kepler equation). Returns false if it did not converge.
MB200_HD inline bool universal_anomaly(double r0, double sig0, double alpha, double mu, double dt, double& s) {
    s = dt / r0;
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
// (x, v) by dt about mu. Returns false if the anomaly did not converge.
MB200_HD inline bool drift_vjp(double mu, const double x[3], const double v[3], double dt, const double lx1[3],
                              const double lv1[3], double lx[3], double lv[3]) {
    const double r0 = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    const double sig0 = x[0] * v[0] + x[1] * v[1] + x[2] * v[2];
    const double vv = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    const double alpha = 2.0 * mu / r0 - vv;
    double s;
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
