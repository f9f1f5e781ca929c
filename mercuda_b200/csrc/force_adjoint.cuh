// Transposed Jacobians of the test-particle accelerations used by the
// adjoints: the Yarkovsky term of mfo_ngf and the changeover-weighted direct
// terms of mfo_drct (HYBRID's interaction force). Each adds J^T la to the
// adjoints gx (positions), gv (velocities) and gyar.
#pragma once
#include <cuda_runtime.h>

namespace mb200 {

// Yarkovsky (mfo_ngf, mercury6_2.for:5106-5153): a = yar t / (r^2 |t|) with
// t = v - (x.v / r^2) x, differentiated in yar even where yar is zero.
__device__ __forceinline__ void yar_vjp(const double3 x, const double3 v, double yar, const double3 la, double3& gx,
                                        double3& gv, double& gyar) {
    const double r2 = x.x * x.x + x.y * x.y + x.z * x.z;
    const double p = x.x * v.x + x.y * v.y + x.z * v.z;
    const double q = p / r2;
    const double3 t = make_double3(v.x - q * x.x, v.y - q * x.y, v.z - q * x.z);
    const double tn = sqrt(t.x * t.x + t.y * t.y + t.z * t.z);
    const double A = la.x * t.x + la.y * t.y + la.z * t.z;
    const double k = yar / (r2 * tn);
    const double kt = A * yar / (r2 * tn * tn * tn);
    const double3 lt = make_double3(k * la.x - kt * t.x, k * la.y - kt * t.y, k * la.z - kt * t.z);
    double lr2 = -A * yar / (r2 * r2 * tn);
    gyar += A / (r2 * tn);
    gv.x += lt.x;
    gv.y += lt.y;
    gv.z += lt.z;
    const double lq = -(lt.x * x.x + lt.y * x.y + lt.z * x.z);
    gx.x -= q * lt.x;
    gx.y -= q * lt.y;
    gx.z -= q * lt.z;
    const double lp = lq / r2;
    lr2 -= lq * p / (r2 * r2);
    gx.x += lp * v.x + 2.0 * lr2 * x.x;
    gx.y += lp * v.y + 2.0 * lr2 * x.y;
    gx.z += lp * v.z + 2.0 * lr2 * x.z;
    gv.x += lp * x.x;
    gv.y += lp * x.y;
    gv.z += lp * x.z;
}

// The changeover factor g(s) of mfo_drct (s^-3 outside rc, 0 inside 0.1 rc,
// K(q) s^-3 between, K = 10q^3 - 15q^4 + 6q^5, q = (s - 0.1 rc) / (0.9 rc))
// and g'(s)/s, for a = -m g(s) d with s = |d|. K'(q) = 30 q^2 (1 - q)^2.
__device__ __forceinline__ void drct_factor_grad(double s2, double rc, double& g, double& g1) {
    const double rc2 = rc * rc;
    if (s2 >= rc2) {
        const double s_1 = 1.0 / sqrt(s2);
        const double s_3 = s_1 * s_1 * s_1;
        g = s_3;
        g1 = -3.0 * s_3 * s_1 * s_1;
        return;
    }
    if (s2 <= 0.01 * rc2) {
        g = 0.0;
        g1 = 0.0;
        return;
    }
    const double s_1 = 1.0 / sqrt(s2);
    const double s = 1.0 / s_1;
    const double s_3 = s_1 * s_1 * s_1;
    const double q = (s - 0.1 * rc) / (0.9 * rc);
    const double q2 = q * q, q3 = q * q2, q4 = q2 * q2, q5 = q2 * q3;
    const double K = 10.0 * q3 - 15.0 * q4 + 6.0 * q5;
    const double Kq = 30.0 * q2 * (1.0 - q) * (1.0 - q);
    g = K * s_3;
    g1 = (Kq / (0.9 * rc) * s_3 - 3.0 * K * s_3 * s_1) * s_1;
}

// a -= m g(s) d, d = x - xb: adds -m [g la + g'(s)/s (d.la) d] to gx.
__device__ __forceinline__ void drct_term_vjp(const double3 x, const double* xb, double m, double rc,
                                              const double3 la, double3& gx) {
    const double dx = x.x - xb[0], dy = x.y - xb[1], dz = x.z - xb[2];
    double g, g1;
    drct_factor_grad(dx * dx + dy * dy + dz * dz, rc, g, g1);
    const double dl = (dx * la.x + dy * la.y + dz * la.z) * g1;
    gx.x -= m * (g * la.x + dl * dx);
    gx.y -= m * (g * la.y + dl * dy);
    gx.z -= m * (g * la.z + dl * dz);
}

}  // namespace mb200
