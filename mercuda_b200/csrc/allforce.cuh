// mfo_all (mercury6_2.for:4506-4571) on the device for the adaptive
// integrators, split as they use it: the massive set (Big bodies and massive
// Small bodies, [3][nsplit] arrays) by one CTA that also writes a table row
// of what every massless particle needs (the indirect sum sx, the oblateness
// reaction acen, the Big bodies' positions and masses), and the massless
// particles from that row. Every sum keeps mfo_grav's order: the indirect sum
// over all bodies by index (massless ones add exactly zero), direct terms with
// Big i outer and j > i inner.
#pragma once
#include "common.cuh"
#include "mvs_device.cuh"

namespace mb200 {

// Force configuration shared by every kernel that evaluates mfo_all.
struct ForceCfg {
    int nbig;      // Big bodies incl. the central body
    int nsplit;    // bodies [0, nsplit) are in the "big" arrays (Big + massive Small)
    int ngflag;
    int pn;
    int obl;
    double jcen[3];
    double m0;
};

// Table row for the particle kernels, in doubles:
// {sx, sy, sz, acen_x, acen_y, acen_z, pad, pad, [x, y, z, m] per Big body}.
constexpr int FT_HEAD = 8;
__host__ __device__ constexpr int force_row(int nb) { return FT_HEAD + 4 * nb; }

// c = 299792458*86400/(AU*0.01) AU/day as mfo_grav/mfo_pr compute it.
__device__ __forceinline__ double light_c() { return 299792458.0 * 86400.0 / (1.495978707e13 * 0.01); }

// The terms of mfo_all after the direct sums: indirect and central terms of
// mfo_grav (with the fused 1PN), then mfo_obl, mfo_ngf, mfo_pr.
// a holds the direct sum; ri = 1/|x|, r3 = ri^3.
__device__ __forceinline__ double3 finish_force(double3 a, const double3 x, const double3 v, double ri, double r3,
                                               const double* T, const ForceCfg& f, double mj, const double* g,
                                               DeviceStatus* st) {
    const double tmp1 = f.m0 * r3;
    if (f.pn == 0) {
        a.x = a.x + T[0] - tmp1 * x.x;
        a.y = a.y + T[1] - tmp1 * x.y;
        a.z = a.z + T[2] - tmp1 * x.z;
    } else {
        const double c = light_c();
        const double light2 = c * c;
        const double rv = 0.0 + x.x * v.x + x.y * v.y + x.z * v.z;
        const double v2 = 0.0 + v.x * v.x + v.y * v.y + v.z * v.z;
        const double ff = tmp1 / light2;
        const double radial = 4.0 * f.m0 * ri - v2;
        a.x = a.x + T[0] - tmp1 * x.x + ff * (radial * x.x + 4.0 * rv * v.x);
        a.y = a.y + T[1] - tmp1 * x.y + ff * (radial * x.y + 4.0 * rv * v.y);
        a.z = a.z + T[2] - tmp1 * x.z + ff * (radial * x.z + 4.0 * rv * v.z);
    }
    if (f.obl) {
        const double3 ao = oblate_accel(x, f.jcen, f.m0);
        a.x = a.x + (ao.x - T[3]);
        a.y = a.y + (ao.y - T[4]);
        a.z = a.z + (ao.z - T[5]);
    }
    if (f.ngflag == 1 || f.ngflag == 3) {
        double3 ng;
        if (!nongrav_accel(x, v, g, ng)) raise_fault(st, FAULT_NGF);
        a.x = a.x + ng.x;
        a.y = a.y + ng.y;
        a.z = a.z + ng.z;
    }
    if (f.ngflag == 2 || f.ngflag == 3) {
        double3 pr = make_double3(0.0, 0.0, 0.0);
        if (!(mj != 0.0 || g[3] == 0.0)) {
            const double c = light_c(), sw = 0.3;
            const double r = sqrt(x.x * x.x + x.y * x.y + x.z * x.z);
            const double vr = (x.x * v.x + x.y * v.y + x.z * v.z) / r;
            const double ff = K2 * g[3] / (r * r);
            pr.x = ff * ((1.0 - (1.0 + sw) * vr / c) * x.x / r - (1.0 + sw) * v.x / c);
            pr.y = ff * ((1.0 - (1.0 + sw) * vr / c) * x.y / r - (1.0 + sw) * v.y / c);
            pr.z = ff * ((1.0 - (1.0 + sw) * vr / c) * x.z / r - (1.0 + sw) * v.z / c);
        }
        a.x = a.x + pr.x;
        a.y = a.y + pr.y;
        a.z = a.z + pr.z;
    }
    if (!isfinite(a.x) || !isfinite(a.y) || !isfinite(a.z)) raise_fault(st, FAULT_NONFINITE);
    return a;
}

// mfo_all for a massless Small body from a table row T (mfo_grav's direct sum
// over the Big bodies in index order, then finish_force).
__device__ __forceinline__ double3 particle_allforce(const double3 x, const double3 v, const double* T, int nb,
                                                     const ForceCfg& f, double mj, const double* g,
                                                     DeviceStatus* st) {
    const double s2c = x.x * x.x + x.y * x.y + x.z * x.z;
    if (s2c <= 0.0) raise_fault(st, FAULT_COINCIDENT);
    const double ri = 1.0 / sqrt(s2c);
    const double r3 = ri * ri * ri;
    double3 a = make_double3(0.0, 0.0, 0.0);
#pragma unroll 1
    for (int b = 0; b < nb; ++b) {
        const double* row = T + FT_HEAD + 4 * b;
        const double dx = x.x - row[0], dy = x.y - row[1], dz = x.z - row[2];
        const double s2 = dx * dx + dy * dy + dz * dz;
        if (s2 <= 0.0) raise_fault(st, FAULT_COINCIDENT);
        const double s_1 = 1.0 / sqrt(s2);
        const double s_3 = s_1 * s_1 * s_1;
        const double tmp1 = s_3 * row[3];
        a.x = a.x - tmp1 * dx;
        a.y = a.y - tmp1 * dy;
        a.z = a.z - tmp1 * dz;
    }
    return finish_force(a, x, v, ri, r3, T, f, mj, g, st);
}

// mfo_all for body k of the massive set, positions X/V [3][ns] in memory,
// T the row being built (sx, acen already in it).
__device__ __forceinline__ double3 massive_allforce(int k, const double* X, const double* V, const double* m,
                                                    const double* ngfbig, const double* T, const ForceCfg& f,
                                                    DeviceStatus* st) {
    const int N = f.nsplit;
    const double3 x = make_double3(X[k], X[N + k], X[2 * N + k]);
    const double3 v = make_double3(V[k], V[N + k], V[2 * N + k]);
    const double s2c = x.x * x.x + x.y * x.y + x.z * x.z;
    if (s2c <= 0.0) raise_fault(st, FAULT_COINCIDENT);
    const double ri = 1.0 / sqrt(s2c);
    const double r3 = ri * ri * ri;
    double3 a = make_double3(0.0, 0.0, 0.0);
    const int last_i = k < f.nbig ? k : f.nbig;
    for (int i = 1; i < last_i; ++i) {  // earlier Big bodies: k is their "j"
        const double dx = x.x - X[i], dy = x.y - X[N + i], dz = x.z - X[2 * N + i];
        const double s2 = dx * dx + dy * dy + dz * dz;
        if (s2 <= 0.0) raise_fault(st, FAULT_COINCIDENT);
        const double s_1 = 1.0 / sqrt(s2);
        const double s_3 = s_1 * s_1 * s_1;
        const double tmp1 = s_3 * m[i];
        a.x = a.x - tmp1 * dx;
        a.y = a.y - tmp1 * dy;
        a.z = a.z - tmp1 * dz;
    }
    if (k < f.nbig)
        for (int j = k + 1; j < N; ++j) {  // later bodies: k is their Big "i"
            const double dx = X[j] - x.x, dy = X[N + j] - x.y, dz = X[2 * N + j] - x.z;
            const double s2 = dx * dx + dy * dy + dz * dz;
            if (s2 <= 0.0) raise_fault(st, FAULT_COINCIDENT);
            const double s_1 = 1.0 / sqrt(s2);
            const double s_3 = s_1 * s_1 * s_1;
            const double tmp2 = s_3 * m[j];
            a.x = a.x + tmp2 * dx;
            a.y = a.y + tmp2 * dy;
            a.z = a.z + tmp2 * dz;
        }
    return finish_force(a, x, v, ri, r3, T, f, m[k], ngfbig + 5 * k, st);
}

// Row head: sx (mfo_grav's indirect sum over every body, in index order; the
// massless particles add exactly zero) and acen (mfo_obl's reaction), from the
// massive set's positions. One thread.
static __device__ void row_head(const double* X, const double* m, const ForceCfg& f, double* T) {
    const int N = f.nsplit;
    double sx = 0.0, sy = 0.0, sz = 0.0, ax = 0.0, ay = 0.0, az = 0.0;
    for (int i = 1; i < N; ++i) {
        const double3 p = make_double3(X[i], X[N + i], X[2 * N + i]);
        const double s2 = p.x * p.x + p.y * p.y + p.z * p.z;
        const double s_1 = 1.0 / sqrt(s2);
        const double r3 = s_1 * s_1 * s_1;
        const double tmp1 = m[i] * r3;
        sx = sx - tmp1 * p.x;
        sy = sy - tmp1 * p.y;
        sz = sz - tmp1 * p.z;
        if (f.obl) {
            const double3 ao = oblate_accel(p, f.jcen, f.m0);
            const double tmp4 = m[i] / f.m0;
            ax = ax - tmp4 * ao.x;
            ay = ay - tmp4 * ao.y;
            az = az - tmp4 * ao.z;
        }
    }
    T[0] = sx; T[1] = sy; T[2] = sz;
    T[3] = ax; T[4] = ay; T[5] = az;
    T[6] = 0.0; T[7] = 0.0;
}

// ---- The massive set's mfo_all by a whole CTA. For sets of up to
// MASSIVE_PAR_MAX bodies the CTA first computes, one term per thread, every
// product the sequential loops above accumulate (massive_terms), so that the
// head (row_head_terms) and each body's acceleration (massive_allforce_terms)
// only add them up in mfo_grav's order: the same roundings in the same order,
// with the sqrt/divide chains of all pairs in flight at once.
constexpr int MASSIVE_PAR_MAX = 32;
// Shared-memory doubles the terms need: body k's q-th direct term at
// [(k * N + q) * 3], then body i's indirect and oblateness-reaction terms at
// [N * N * 3 + i * 6].
__host__ __device__ constexpr int massive_par_scratch(int N) { return N <= MASSIVE_PAR_MAX ? N * N * 3 + N * 6 : 0; }

// Number of body k's direct terms that come from earlier Big bodies (they are
// subtracted); later bodies' terms follow (they are added).
__device__ __forceinline__ int massive_earlier(int k, const ForceCfg& f) { return (k < f.nbig ? k : f.nbig) - 1; }

static __device__ void massive_terms(const double* X, const double* m, const ForceCfg& f, double* PT, DeviceStatus* st) {
    const int N = f.nsplit;
    for (int q = threadIdx.x; q < N * N; q += blockDim.x) {
        const int k = q / N, o = q - k * N;
        if (k < 1 || o < 1 || o == k) continue;
        const int ne = massive_earlier(k, f);
        int slot;
        double dx, dy, dz;
        if (o <= ne) {  // earlier Big body o: k is its "j"
            slot = o - 1;
            dx = X[k] - X[o]; dy = X[N + k] - X[N + o]; dz = X[2 * N + k] - X[2 * N + o];
        } else if (k < f.nbig && o > k) {  // later body o: k is its Big "i"
            slot = ne + (o - k - 1);
            dx = X[o] - X[k]; dy = X[N + o] - X[N + k]; dz = X[2 * N + o] - X[2 * N + k];
        } else {
            continue;
        }
        const double s2 = dx * dx + dy * dy + dz * dz;
        if (s2 <= 0.0) raise_fault(st, FAULT_COINCIDENT);
        const double s_1 = 1.0 / sqrt(s2);
        const double s_3 = s_1 * s_1 * s_1;
        const double t = s_3 * m[o];
        double* out = PT + ((size_t)k * N + slot) * 3;
        out[0] = t * dx;
        out[1] = t * dy;
        out[2] = t * dz;
    }
    double* HT = PT + (size_t)N * N * 3;
    for (int i = 1 + threadIdx.x; i < N; i += blockDim.x) {
        const double3 p = make_double3(X[i], X[N + i], X[2 * N + i]);
        const double s2 = p.x * p.x + p.y * p.y + p.z * p.z;
        const double s_1 = 1.0 / sqrt(s2);
        const double r3 = s_1 * s_1 * s_1;
        const double tmp1 = m[i] * r3;
        double* out = HT + (size_t)i * 6;
        out[0] = tmp1 * p.x;
        out[1] = tmp1 * p.y;
        out[2] = tmp1 * p.z;
        if (f.obl) {
            const double3 ao = oblate_accel(p, f.jcen, f.m0);
            const double tmp4 = m[i] / f.m0;
            out[3] = tmp4 * ao.x;
            out[4] = tmp4 * ao.y;
            out[5] = tmp4 * ao.z;
        }
    }
}

// row_head from the terms (one thread).
static __device__ void row_head_terms(const double* PT, const ForceCfg& f, double* T) {
    const int N = f.nsplit;
    const double* HT = PT + (size_t)N * N * 3;
    double sx = 0.0, sy = 0.0, sz = 0.0, ax = 0.0, ay = 0.0, az = 0.0;
    for (int i = 1; i < N; ++i) {
        const double* t = HT + (size_t)i * 6;
        sx = sx - t[0];
        sy = sy - t[1];
        sz = sz - t[2];
        if (f.obl) {
            ax = ax - t[3];
            ay = ay - t[4];
            az = az - t[5];
        }
    }
    T[0] = sx; T[1] = sy; T[2] = sz;
    T[3] = ax; T[4] = ay; T[5] = az;
    T[6] = 0.0; T[7] = 0.0;
}

// massive_allforce from the terms.
__device__ __forceinline__ double3 massive_allforce_terms(int k, const double* X, const double* V, const double* m,
                                                          const double* ngfbig, const double* T, const ForceCfg& f,
                                                          const double* PT, DeviceStatus* st) {
    const int N = f.nsplit;
    const double3 x = make_double3(X[k], X[N + k], X[2 * N + k]);
    const double3 v = make_double3(V[k], V[N + k], V[2 * N + k]);
    const double s2c = x.x * x.x + x.y * x.y + x.z * x.z;
    if (s2c <= 0.0) raise_fault(st, FAULT_COINCIDENT);
    const double ri = 1.0 / sqrt(s2c);
    const double r3 = ri * ri * ri;
    double3 a = make_double3(0.0, 0.0, 0.0);
    const int ne = massive_earlier(k, f);
    const int nl = k < f.nbig ? N - k - 1 : 0;
    const double* t = PT + (size_t)k * N * 3;
    for (int q = 0; q < ne; ++q, t += 3) {
        a.x = a.x - t[0];
        a.y = a.y - t[1];
        a.z = a.z - t[2];
    }
    for (int q = 0; q < nl; ++q, t += 3) {
        a.x = a.x + t[0];
        a.y = a.y + t[1];
        a.z = a.z + t[2];
    }
    return finish_force(a, x, v, ri, r3, T, f, m[k], ngfbig + 5 * k, st);
}

}  // namespace mb200
