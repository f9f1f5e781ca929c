// Device pieces of the MVS map shared by the big-body and particle kernels:
// encounter minimum, x-y bounding box, non-gravitational force, oblateness,
// and the event-record writer.
#pragma once
#include "common.cuh"
#include "mvs.cuh"

namespace mb200 {

// mce_min (mercury6_2.for:1572-1622): cubic-interpolated minimum of the squared
// separation over a step of length h, given its end values and derivatives.
__device__ __forceinline__ void encounter_minimum(double d0, double d1, double d0t, double d1t, double h,
                                                  double& d2min, double& tmin) {
    if (d0t * h > 0.0 || d1t * h < 0.0) {
        if (d0 <= d1) { d2min = d0; tmin = -h; }
        else { d2min = d1; tmin = 0.0; }
        return;
    }
    double temp = 6.0 * (d0 - d1);
    const double a = temp + 3.0 * h * (d0t + d1t);
    const double b = temp + 2.0 * h * (d0t + 2.0 * d1t);
    const double c = h * d1t;
    const double disc = b * b - 4.0 * a * c;
    temp = -(0.5 * (b + copysign(sqrt(disc > 0.0 ? disc : 0.0), b)));
    double tau = (temp == 0.0) ? 0.0 : c / temp;
    tau = tau < 0.0 ? tau : 0.0;
    tau = tau > -1.0 ? tau : -1.0;
    tmin = tau * h;
    temp = 1.0 + tau;
    d2min = tau * tau * ((3.0 + 2.0 * tau) * d0 + temp * h * d0t) +
            temp * temp * ((1.0 - 2.0 * tau) * d1 + tau * h * d1t);
    d2min = d2min > 0.0 ? d2min : 0.0;
}

// One coordinate of mce_box (mercury6_2.for:997-1040): extent of a body over
// the step with the turning point interpolated when the velocity changes sign.
__device__ __forceinline__ void box_extent(double a0, double a1, double u0, double u1, double h,
                                           double& lo, double& hi) {
    lo = a0 < a1 ? a0 : a1;
    hi = a0 > a1 ? a0 : a1;
    if ((u0 < 0.0 && u1 > 0.0) || (u0 > 0.0 && u1 < 0.0)) {
        const double temp = (u0 * a1 - u1 * a0 - 0.5 * h * u0 * u1) / (u0 - u1);
        lo = lo < temp ? lo : temp;
        hi = hi > temp ? hi : temp;
    }
}

// mfo_ngf for one body (mercury6_2.for:5106-5153): Marsden A1/A2/A3 with the
// 88 AU^2 cutoff and the inverse-square transverse Yarkovsky term.
// g = {A1, A2, A3, beta, yar}. Returns false where the Fortran calls fail().
__device__ __forceinline__ bool nongrav_accel(const double3 p, const double3 u, const double* g,
                                              double3& a) {
    a = make_double3(0.0, 0.0, 0.0);
    if (g[0] == 0.0 && g[1] == 0.0 && g[2] == 0.0 && g[4] == 0.0) return true;
    const double r2 = 0.0 + p.x * p.x + p.y * p.y + p.z * p.z;
    const double r = sqrt(r2);
    const double rv = (0.0 + p.x * u.x + p.y * u.y + p.z * u.z) / r2;
    const double tx = u.x - rv * p.x, ty = u.y - rv * p.y, tz = u.z - rv * p.z;
    const double tn = sqrt(tx * tx + ty * ty + tz * tz);
    const bool any = g[0] != 0.0 || g[1] != 0.0 || g[2] != 0.0;
    const bool big = fabs(g[0]) > 1e-7 || fabs(g[1]) > 1e-7 || fabs(g[2]) > 1e-7;
    if (any && (r2 < 88.0 || big)) {
        const double q = r * 0.3561253561253561;
        const double gg = 0.111262 * pow(q, -2.15) * pow(1.0 + pow(q, 5.093), -4.6142);
        a.x = g[0] * gg / r * p.x;
        a.y = g[0] * gg / r * p.y;
        a.z = g[0] * gg / r * p.z;
        if (g[1] != 0.0) {
            if (tn == 0.0) return false;
            const double f = g[1] * gg / tn;
            a.x = a.x + f * tx; a.y = a.y + f * ty; a.z = a.z + f * tz;
        }
        if (g[2] != 0.0) {
            const double nx = p.y * u.z - p.z * u.y, ny = p.z * u.x - p.x * u.z, nz = p.x * u.y - p.y * u.x;
            const double nn = sqrt(nx * nx + ny * ny + nz * nz);
            if (nn == 0.0) return false;
            const double f = g[2] * gg / nn;
            a.x = a.x + f * nx; a.y = a.y + f * ny; a.z = a.z + f * nz;
        }
    }
    if (g[4] != 0.0) {
        if (tn == 0.0) return false;
        const double f = g[4] / (r2 * tn);
        a.x = a.x + f * tx; a.y = a.y + f * ty; a.z = a.z + f * tz;
    }
    return true;
}

// Acceleration of one body from the central body's J2/J4/J6 (mfo_obl,
// mercury6_2.for:5196-5218); jcen = J2 R^2, J4 R^4, J6 R^6.
__device__ __forceinline__ double3 oblate_accel(const double3 p, const double* jcen, double m0) {
    const double r2 = p.x * p.x + p.y * p.y + p.z * p.z;
    const double r_1 = 1.0 / sqrt(r2);
    const double r_2 = r_1 * r_1;
    const double r_3 = r_2 * r_1;
    const double jr2 = jcen[0] * r_2;
    const double jr4 = jcen[1] * r_2 * r_2;
    const double jr6 = jcen[2] * r_2 * r_2 * r_2;
    const double u2 = p.z * p.z * r_2;
    const double u4 = u2 * u2;
    const double u6 = u4 * u2;
    const double tmp1 = m0 * r_3;
    const double tmp2 = jr2 * (7.5 * u2 - 1.5) + jr4 * (39.375 * u4 - 26.25 * u2 + 1.875) +
                        jr6 * (187.6875 * u6 - 216.5625 * u4 + 59.0625 * u2 - 2.1875);
    const double tmp3 = jr2 * 3.0 + jr4 * (17.5 * u2 - 7.5) + jr6 * (86.625 * u4 - 78.75 * u2 + 13.125);
    return make_double3(p.x * tmp1 * tmp2, p.y * tmp1 * tmp2, p.z * tmp1 * (tmp2 - tmp3));
}

// State of one body at both ends of the drift, as mce_stat sees it.
struct PairEnds {
    double3 x0, v0, x1, v1;
};

// Classification of one pair by mce_stat's test (mercury6_2.for:1815-1908).
struct PairClass {
    double d2min, tmin;
    int kind, now;
};

// mce_stat for one pair (i Big, j after it): true when the pair is a close-
// encounter minimum (kind bit 1), a near miss (2) or a collision (4).
__device__ __forceinline__ bool pair_classify(const PairEnds& I, const PairEnds& J, double rce_i, double rce_j,
                                              double rphys_i, double rphys_j, double h, PairClass& pc) {
    const double dx0 = I.x0.x - J.x0.x, dy0 = I.x0.y - J.x0.y, dz0 = I.x0.z - J.x0.z;
    const double du0 = I.v0.x - J.v0.x, dv0 = I.v0.y - J.v0.y, dw0 = I.v0.z - J.v0.z;
    const double d0t = (dx0 * du0 + dy0 * dv0 + dz0 * dw0) * 2.0;
    const double dx1 = I.x1.x - J.x1.x, dy1 = I.x1.y - J.x1.y, dz1 = I.x1.z - J.x1.z;
    const double du1 = I.v1.x - J.v1.x, dv1 = I.v1.y - J.v1.y, dw1 = I.v1.z - J.v1.z;
    const double d1t = (dx1 * du1 + dy1 * dv1 + dz1 * dw1) * 2.0;
    const double d0 = dx0 * dx0 + dy0 * dy0 + dz0 * dz0;
    const double d1 = dx1 * dx1 + dy1 * dy1 + dz1 * dz1;
    double d2min, tmin;
    encounter_minimum(d0, d1, d0t, d1t, h, d2min, tmin);
    double d2ce = rce_i > rce_j ? rce_i : rce_j;
    double d2hit = rphys_i + rphys_j;
    d2ce = d2ce * d2ce;
    d2hit = d2hit * d2hit;
    const double d2near = d2hit * 4.0;
    const bool clo = (d2min <= d2ce && d0t * h <= 0.0 && d1t * h >= 0.0) || (d2min <= d2hit);
    const bool near = d2min <= d2near;
    pc.d2min = d2min;
    pc.tmin = tmin;
    pc.kind = (clo ? EV_CLOSE : 0) | (near ? EV_NEAR : 0) | (d2min <= d2hit ? EV_HIT : 0);
    pc.now = d1 <= d2hit ? 1 : 0;
    return clo || near;
}

// Writes the merged record of a classified pair straight into its slot:
// ids 1-based with the more massive Big body first (`swap` lists J first),
// time holding tmin (the caller's host adds the step's end time), states
// linearly interpolated to tmin as mce_stat:1869-1882 does.
__device__ __forceinline__ void pair_record(MercuryEvent* dst, const PairEnds& I, const PairEnds& J,
                                            const PairClass& pc, double hm1, int id_i, int id_j, bool swap) {
    const PairEnds& A = swap ? J : I;
    const PairEnds& B = swap ? I : J;
    const double tmp0 = -(pc.tmin * hm1);
    const double tmp1 = 1.0 + pc.tmin * hm1;
    double2* d = reinterpret_cast<double2*>(dst);
    int4 head = make_int4(swap ? id_j : id_i, swap ? id_i : id_j, pc.kind, pc.now);
    *reinterpret_cast<int4*>(dst) = head;
    d[1] = make_double2(sqrt(pc.d2min > 0.0 ? pc.d2min : 0.0), pc.tmin);
    d[2] = make_double2(tmp0 * A.x0.x + tmp1 * A.x1.x, tmp0 * A.x0.y + tmp1 * A.x1.y);
    d[3] = make_double2(tmp0 * A.x0.z + tmp1 * A.x1.z, tmp0 * A.v0.x + tmp1 * A.v1.x);
    d[4] = make_double2(tmp0 * A.v0.y + tmp1 * A.v1.y, tmp0 * A.v0.z + tmp1 * A.v1.z);
    d[5] = make_double2(tmp0 * B.x0.x + tmp1 * B.x1.x, tmp0 * B.x0.y + tmp1 * B.x1.y);
    d[6] = make_double2(tmp0 * B.x0.z + tmp1 * B.x1.z, tmp0 * B.v0.x + tmp1 * B.v1.x);
    d[7] = make_double2(tmp0 * B.v0.y + tmp1 * B.v1.y, tmp0 * B.v0.z + tmp1 * B.v1.z);
}

// mce_cent for one body (mercury6_2.for:1091-1160), algor != 11, split into
// the start-of-step quantities (|x0|^2, v0.x0, |x0 x v0|^2, |v0|^2) and the
// test at the end of the step, so that a caller may keep four numbers instead
// of the start state. Returns true on an impact with the entry time offset
// `temp` from the step's start; the event time is (time_end - h) + temp.
struct CentralStart {
    double rr0, rv0, h2, v2;
};

__device__ __forceinline__ CentralStart central_start(const double3 p0, const double3 u0) {
    CentralStart c;
    c.rr0 = p0.x * p0.x + p0.y * p0.y + p0.z * p0.z;
    c.rv0 = u0.x * p0.x + u0.y * p0.y + u0.z * p0.z;
    const double hx = p0.y * u0.z - p0.z * u0.y;
    const double hy = p0.z * u0.x - p0.x * u0.z;
    const double hz = p0.x * u0.y - p0.y * u0.x;
    c.v2 = u0.x * u0.x + u0.y * u0.y + u0.z * u0.z;
    c.h2 = hx * hx + hy * hy + hz * hz;
    return c;
}

static __device__ __noinline__ bool central_finish(const CentralStart c, const double3 p1, const double3 u1, double mcen,
                                            double mj, double h, double rcen, double& temp) {
    const double rcen2 = rcen * rcen;
    const double rr1 = p1.x * p1.x + p1.y * p1.y + p1.z * p1.z;
    const double rv1 = u1.x * p1.x + u1.y * p1.y + u1.z * p1.z;
    const double rmin = c.rr0 < rr1 ? c.rr0 : rr1;
    if (!((c.rv0 * h <= 0.0 && rv1 * h >= 0.0) || rmin <= rcen2)) return false;
    const double p = c.h2 / (mcen + mj);
    const double r0 = sqrt(c.rr0);
    double t = 1.0 + p * (c.v2 / (mcen + mj) - 2.0 / r0);
    const double e = sqrt(t > 0.0 ? t : 0.0);
    const double q = p / (1.0 + e);
    if (!(q <= rcen)) return false;
    t = 0.0;
    if (e > 0.0 && e < 1.0) {
        const double a = q / (1.0 - e);
        double c1 = (1.0 - rcen / a) / e, c2 = (1.0 - r0 / a) / e;
        c1 = c1 < 1.0 ? c1 : 1.0; c1 = c1 > -1.0 ? c1 : -1.0;
        c2 = c2 < 1.0 ? c2 : 1.0; c2 = c2 > -1.0 ? c2 : -1.0;
        const double uhit = copysign(acos(c1), -h);
        const double uu0 = copysign(acos(c2), c.rv0);
        const double mhit = uhit - e * sin(uhit);
        const double m0 = uu0 - e * sin(uu0);
        t = (mhit - m0) / sqrt((mcen + mj) / (a * a * a));
    } else if (e > 1.0) {
        const double a = q / (e - 1.0);
        double c1 = (1.0 + rcen / a) / e, c2 = (1.0 + r0 / a) / e;
        c1 = c1 > 1.0 ? c1 : 1.0;
        c2 = c2 > 1.0 ? c2 : 1.0;
        const double uhit = copysign(acosh(c1), -h);
        const double uu0 = copysign(acosh(c2), c.rv0);
        const double mhit = e * sinh(uhit) - uhit;
        const double m0 = e * sinh(uu0) - uu0;
        t = (mhit - m0) / sqrt((mcen + mj) / (a * a * a));
    } else if (e == 1.0 && q > 0.0) {
        const double g1 = rcen / q - 1.0, g2 = r0 / q - 1.0;
        const double uhit = copysign(sqrt(g1 > 0.0 ? g1 : 0.0), -h);
        const double uu0 = copysign(sqrt(g2 > 0.0 ? g2 : 0.0), c.rv0);
        t = sqrt(2.0 * (q * q * q) / (mcen + mj)) *
            (uhit + (uhit * uhit * uhit) / 3.0 - uu0 - (uu0 * uu0 * uu0) / 3.0);
    }
    if (q == 0.0 && rr1 != c.rr0) {
        double w = (r0 - rcen) / (r0 - sqrt(rr1));
        w = w < 1.0 ? w : 1.0;
        w = w > 0.0 ? w : 0.0;
        t = h * w;
    }
    temp = t;
    return true;
}

__device__ __forceinline__ bool central_impact(const double3 p0, const double3 u0, const double3 p1,
                                               const double3 u1, double mcen, double mj, double h,
                                               double rcen, double& temp) {
    return central_finish(central_start(p0, u0), p1, u1, mcen, mj, h, rcen, temp);
}

// 128-byte record store as eight 16-byte writes.
__device__ __forceinline__ void store_event(MercuryEvent* dst, const MercuryEvent& e) {
    const double2* s = reinterpret_cast<const double2*>(&e);
    double2* d = reinterpret_cast<double2*>(dst);
#pragma unroll
    for (int k = 0; k < 8; ++k) d[k] = s[k];
}

// mfo_mvs for one Small body (mercury6_2.for:5034-5060) plus mfo_ngf, i.e. the
// total acceleration (angf + 0) + a of the kick; T is a force table and g(c)
// returns the body's c-th non-gravitational coefficient.
template <bool NGF, bool OBL, class G>
__device__ __forceinline__ double3 small_body_force(const double3 x, const double3 v_ngf, G g, const double* T,
                                                    int nb, const double* jcen, double mu, DeviceStatus* st) {
    double3 a3 = make_double3(0.0, 0.0, 0.0);
#pragma unroll 1
    for (int b = 0; b < nb; ++b) {
        const double* row = T + TAB_HEAD + b * TAB_BODY;
        const double dx = x.x - row[0], dy = x.y - row[1], dz = x.z - row[2];
        const double s2 = dx * dx + dy * dy + dz * dz;
        const double s_1 = 1.0 / sqrt(s2);
        const double s_3 = s_1 * s_1 * s_1;
        const double faci = row[3] * s_3;
        a3.x = a3.x - faci * dx;
        a3.y = a3.y - faci * dy;
        a3.z = a3.z - faci * dz;
    }
    double3 a = make_double3(T[0] + a3.x, T[1] + a3.y, T[2] + a3.z);
    if (OBL) {
        const double3 ao = oblate_accel(x, jcen, mu);
        a.x = a.x + (ao.x - T[3]);
        a.y = a.y + (ao.y - T[4]);
        a.z = a.z + (ao.z - T[5]);
    }
    if (NGF) {
        double gc[5];
        for (int c = 0; c < 5; ++c) gc[c] = g(c);
        double3 ng;
        if (!nongrav_accel(x, v_ngf, gc, ng)) raise_fault(st, 2);
        a.x = ng.x + 0.0 + a.x;
        a.y = ng.y + 0.0 + a.y;
        a.z = ng.z + 0.0 + a.z;
    }
    if (!isfinite(a.x) || !isfinite(a.y) || !isfinite(a.z)) raise_fault(st, 1);
    return a;
}

}  // namespace mb200
