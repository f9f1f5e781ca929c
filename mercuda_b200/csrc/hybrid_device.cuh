// Device functions of the HYBRID step shared by its kernels and the HYBRID
// adjoint: the changeover factor of mfo_drct and the particles' kick force.
#pragma once
#include "hybrid.cuh"
#include "mvs_device.cuh"

namespace mb200 {

// mfo_drct's changeover factor (mercury6_2.for:4733-4750): s^-3 outside rc,
// 0 inside 0.1 rc, K(q) s^-3 with K = 10q^3 - 15q^4 + 6q^5 between.
__device__ __forceinline__ double drct_factor(double s2, double rc) {
    const double rc2 = rc * rc;
    if (s2 >= rc2) {
        const double s_1 = 1.0 / sqrt(s2);
        return s_1 * s_1 * s_1;
    }
    if (s2 <= 0.01 * rc2) return 0.0;
    const double s_1 = 1.0 / sqrt(s2);
    const double s = 1.0 / s_1;
    const double s_3 = s_1 * s_1 * s_1;
    const double q = (s - 0.1 * rc) / (0.9 * rc);
    const double q2 = q * q, q3 = q * q2, q4 = q2 * q2, q5 = q2 * q3;
    return (10.0 * q3 - 15.0 * q4 + 6.0 * q5) * s_3;
}

// (angf + 0) + a of mdt_hy's kick for a massless particle against a force
// row T: mfo_hy's direct terms from every Big body, oblateness, mfo_ngf.
__device__ __forceinline__ double3 particle_hy_accel(const HyArgs& A, const double3 x, const double3 v,
                                                     double rcrit_p, const double* g, const double* T) {
    const int nb = A.nbig - 1;
    double3 a = make_double3(0.0, 0.0, 0.0);
#pragma unroll 1
    for (int b = 0; b < nb; ++b) {
        const double* row = T + HY_HEAD + b * HY_FORCE_BODY;
        const double dx = x.x - row[0], dy = x.y - row[1], dz = x.z - row[2];
        const double tmp2 = drct_factor(dx * dx + dy * dy + dz * dz, fmax(row[4], rcrit_p));
        const double faci = tmp2 * row[3];
        a.x = a.x - faci * dx;
        a.y = a.y - faci * dy;
        a.z = a.z - faci * dz;
    }
    if (A.obl) {
        const double3 ao = oblate_accel(x, A.jcen, A.m0);
        a.x = a.x + ao.x - T[3];
        a.y = a.y + ao.y - T[4];
        a.z = a.z + ao.z - T[5];
    }
    if (A.ngflag == 1 || A.ngflag == 3) {
        double3 ng;
        if (!nongrav_accel(x, v, g, ng)) raise_fault(A.status, FAULT_NGF);
        a.x = ng.x + 0.0 + a.x;
        a.y = ng.y + 0.0 + a.y;
        a.z = ng.z + 0.0 + a.z;
    }
    if (!isfinite(a.x) || !isfinite(a.y) || !isfinite(a.z)) raise_fault(A.status, FAULT_NONFINITE);
    return a;
}

}  // namespace mb200
