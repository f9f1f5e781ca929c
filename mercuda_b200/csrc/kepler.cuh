// Universal-variable Kepler drift for one body, FP64, on the device.
//
// Restates SWIFT's drift_* routines as they appear in mercury6_2.for:7602-8330
// (Levison & Duncan) and mco_sine (mercury6_2.for:2940-2972), keeping every
// statement's operand order so that, with --fmad=false, each result rounds as
// the Fortran CPU build rounds it. The paths are: the elliptic small-step
// solver drift_kepmd when dm^2 <= 0.16, e^2 <= 0.36 and e^2 dm^2 < 0.0016;
// otherwise drift_kepu (seed from drift_kepu_guess, up to 7 quartic Newton
// iterations, then at most 401 Laguerre iterations); drift_one retries a
// failed drift as ten substeps and keeps the partial result, as every caller
// in the reference does.
#pragma once
#include "common.cuh"

namespace mb200 {

// drift_kepu_stumpff: argument quartering, degree-6 series, doubling back.
// Any finite argument falls below 0.1 within about 520 quarterings; the cap
// only stops a non-finite argument (which then yields a non-finite result and
// a failed drift) from looping forever.
constexpr int STUMPFF_MAX_QUARTERINGS = 2000;
__device__ __forceinline__ void stumpff(double x, double& c0, double& c1, double& c2, double& c3) {
    int n = 0;
    while (fabs(x) >= 0.1 && n < STUMPFF_MAX_QUARTERINGS) {
        n = n + 1;
        x = x * 0.25;
    }
    const double x2 = x * x, x3 = x * x2, x4 = x2 * x2, x5 = x2 * x3, x6 = x3 * x3;
    c2 = 1.147074559772972e-11 * x6 - 2.087675698786810e-9 * x5 + 2.755731922398589e-7 * x4 -
         2.480158730158730e-5 * x3 + 1.388888888888889e-3 * x2 - 4.166666666666667e-2 * x + 0.5;
    c3 = 7.647163731819816e-13 * x6 - 1.605904383682161e-10 * x5 + 2.505210838544172e-8 * x4 -
         2.755731922398589e-6 * x3 + 1.984126984126984e-4 * x2 - 8.333333333333333e-3 * x +
         1.666666666666667e-1;
    c1 = 1.0 - x * c3;
    c0 = 1.0 - x * c2;
#pragma unroll 1
    for (int i = n; i >= 1; --i) {
        c3 = (c2 + c0 * c3) * 0.25;
        c2 = c1 * c1 * 0.5;
        c1 = c0 * c1;
        c0 = 2.0 * c0 * c0 - 1.0;
    }
}

// drift_kepu_fchk: residual of the universal Kepler equation at s.
__device__ __forceinline__ double kepu_residual(double dt, double r0, double mu, double alpha, double u,
                                                double s) {
    double c0, c1, c2, c3;
    stumpff(s * s * alpha, c0, c1, c2, c3);
    c1 = c1 * s;
    c2 = c2 * s * s;
    c3 = c3 * s * s * s;
    return r0 * c1 + u * c2 + mu * c3 - dt;
}

// drift_kepu_p3solve: Cardano seed for alpha <= 0. Returns false when no real root.
static __device__ __noinline__ bool kepu_cubic_seed(double dt, double r0, double mu, double alpha, double u,
                                             double& s) {
    const double denom = (mu - alpha * r0) / 6.0;
    const double a2 = 0.5 * u / denom;
    const double a1 = r0 / denom;
    const double a0 = -dt / denom;
    const double q = (a1 - a2 * a2 / 3.0) / 3.0;
    const double r = (a1 * a2 - 3.0 * a0) / 6.0 - pow(a2, 3.0) / 27.0;
    const double sq2 = pow(q, 3.0) + r * r;
    if (sq2 >= 0.0) {
        const double sq = sqrt(sq2), third = 1.0 / 3.0;
        const double p1 = (r + sq) <= 0.0 ? -pow(-(r + sq), third) : pow(r + sq, third);
        const double p2 = (r - sq) <= 0.0 ? -pow(-(r - sq), third) : pow(r - sq, third);
        s = p1 + p2 - a2 / 3.0;
        return true;
    }
    s = 0.0;
    return false;
}

// drift_kepu_guess (with mco_sine for the elliptic long-step seed).
__device__ __forceinline__ double kepu_guess(double dt, double r0, double mu, double alpha, double u) {
    if (alpha > 0.0) {
        if (dt / r0 <= 0.4) return dt / r0 - (dt * dt * u) / (2.0 * r0 * r0 * r0);
        const double a = mu / alpha;
        const double en = sqrt(mu / (a * a * a));
        const double ec = 1.0 - r0 / a;
        const double es = u / (en * a * a);
        const double e = sqrt(ec * ec + es * es);
        double y = en * dt - es;
        // mco_sine
        const double pi = 3.141592653589793, twopi = 2.0 * pi;
        if (y > 0.0) y = fmod(y, twopi);
        else y = fmod(y, twopi) + twopi;
        const double cy = cos(y);
        const double sy = (y > pi) ? -sqrt(1.0 - cy * cy) : sqrt(1.0 - cy * cy);
        const double sigma = copysign(1.0, es * cy + ec * sy);
        const double x = y + sigma * 0.85 * e;
        return x / sqrt(alpha);
    }
    double s;
    if (!kepu_cubic_seed(dt, r0, mu, alpha, u, s)) s = dt / r0;
    return s;
}

// drift_kepu_new: quartic Newton, at most 7 passes. Returns true on convergence.
__device__ __forceinline__ bool kepu_newton(double& s, double dt, double r0, double mu, double alpha,
                                            double u, double& fp, double& c1, double& c2, double& c3) {
    const double tol = DANBYB * DANBYB;
#pragma unroll 1
    for (int nc = 0; nc <= 6; ++nc) {
        const double s2 = s * s;
        double c0;
        stumpff(s2 * alpha, c0, c1, c2, c3);
        c1 = c1 * s;
        c2 = c2 * s2;
        c3 = c3 * s * s2;
        const double f = r0 * c1 + u * c2 + mu * c3 - dt;
        fp = r0 * c0 + u * c1 + mu * c2;
        const double fpp = (mu - r0 * alpha) * c1 + u * c0;
        const double fppp = (mu - r0 * alpha) * c0 - u * alpha * c1;
        double ds = -(f / fp);
        ds = -(f / (fp + 0.5 * ds * fpp));
        ds = -(f / (fp + 0.5 * ds * fpp + ds * ds * fppp * 0.1666666666666667));
        s = s + ds;
        const double fdt = f / dt;
        if (fdt * fdt < tol) return true;
    }
    return false;
}

// drift_kepu_lag: Laguerre iteration (n = 5), at most 401 passes; rarely taken.
static __device__ __noinline__ bool kepu_laguerre(double& s, double dt, double r0, double mu, double alpha,
                                           double u, double& fp, double& c1, double& c2, double& c3) {
    const double ln = 5.0, tol = DANBYB * DANBYB;
#pragma unroll 1
    for (int nc = 0; nc <= 400; ++nc) {
        double c0;
        stumpff(s * s * alpha, c0, c1, c2, c3);
        c1 = c1 * s;
        c2 = c2 * s * s;
        c3 = c3 * s * s * s;
        const double f = r0 * c1 + u * c2 + mu * c3 - dt;
        fp = r0 * c0 + u * c1 + mu * c2;
        const double fpp = (-40.0 * alpha + mu) * c1 + u * c0;
        const double ds = -(ln * f / (fp + copysign(1.0, fp) *
                                                sqrt(fabs((ln - 1.0) * (ln - 1.0) * fp * fp -
                                                          (ln - 1.0) * ln * f * fpp))));
        s = s + ds;
        const double fdt = f / dt;
        if (fdt * fdt < tol) return true;
    }
    return false;
}

// drift_kepu: guess, Newton, and on failure the better of the two seeds for Laguerre.
__device__ __forceinline__ bool kepu(double dt, double r0, double mu, double alpha, double u, double& fp,
                                     double& c1, double& c2, double& c3) {
    double s = kepu_guess(dt, r0, mu, alpha, u);
    const double st = s;
    if (kepu_newton(s, dt, r0, mu, alpha, u, fp, c1, c2, c3)) return true;
    const double fo = kepu_residual(dt, r0, mu, alpha, u, st);
    const double fn = kepu_residual(dt, r0, mu, alpha, u, s);
    if (fabs(fo) < fabs(fn)) s = st;
    return kepu_laguerre(s, dt, r0, mu, alpha, u, fp, c1, c2, c3);
}

// Series for sin x of drift_kepmd (Horner form over 11!).
__device__ __forceinline__ double kepmd_sine(double x) {
    const double y = x * x;
    return x * (39916800.0 - y * (6652800.0 - y * (332640.0 - y * (7920.0 - y * (110.0 - y))))) /
           39916800.0;
}

// drift_dan. State (p, w) is updated in place; returns false (state untouched)
// when neither solver converged, which makes drift_one substep.
__device__ __forceinline__ bool drift_dan(double mu, double3& p, double3& w, double dt0) {
    double dt = dt0;
    const double r0 = sqrt(p.x * p.x + p.y * p.y + p.z * p.z);
    const double v0s = w.x * w.x + w.y * w.y + w.z * w.z;
    const double u = p.x * w.x + p.y * w.y + p.z * w.z;
    const double alpha = 2.0 * mu / r0 - v0s;
    double f, g, fdot, gdot;
    bool done = false;
    if (alpha > 0.0) {
        const double a = mu / alpha;
        const double asq = a * a;
        const double en = sqrt(mu / (a * asq));
        const double ec = 1.0 - r0 / a;
        const double es = u / (en * asq);
        const double esq = ec * ec + es * es;
        const double dm = dt * en - double(int(dt * en / TWOPI_SWIFT)) * TWOPI_SWIFT;
        dt = dm / en;
        if (!((dm * dm > 0.16) || (esq > 0.36)) && esq * dm * dm < 0.0016) {
            // drift_kepmd: cubic seed, one quartic Newton correction.
            const double fac1 = 1.0 / (1.0 - ec);
            const double q = fac1 * dm;
            const double fac2 = es * es * fac1 - ec / 3.0;
            double x = q * (1.0 - 0.5 * fac1 * q * (es - q * fac2));
            double s = kepmd_sine(x);
            double c = sqrt(1.0 - s * s);
            {
                const double ff = x - ec * s + es * (1.0 - c) - dm;
                const double ffp = 1.0 - ec * c + es * s;
                const double ffpp = ec * s + es * c;
                const double ffppp = ec * c - es * s;
                double dx = -(ff / ffp);
                dx = -(ff / (ffp + 0.5 * dx * ffpp));
                dx = -(ff / (ffp + 0.5 * dx * ffpp + 0.16666666666666666 * dx * dx * ffppp));
                x = x + dx;
            }
            s = kepmd_sine(x);
            c = sqrt(1.0 - s * s);
            const double fchk = (x - ec * s + es * (1.0 - c) - dm);
            if (fchk * fchk > DANBYB) return false;
            const double fp = 1.0 - ec * c + es * s;
            f = (a / r0) * (c - 1.0) + 1.0;
            g = dt + (s - x) / en;
            fdot = -(a / (r0 * fp)) * en * s;
            gdot = (c - 1.0) / fp + 1.0;
            done = true;
        }
    }
    if (!done) {
        double fp, c1, c2, c3;
        if (!kepu(dt, r0, mu, alpha, u, fp, c1, c2, c3)) return false;
        f = 1.0 - (mu / r0) * c2;
        g = dt - mu * c3;
        fdot = -(mu / (fp * r0)) * c1;
        gdot = 1.0 - (mu / fp) * c2;
    }
    const double3 p1 = make_double3(p.x * f + w.x * g, p.y * f + w.y * g, p.z * f + w.z * g);
    const double3 w1 = make_double3(p.x * fdot + w.x * gdot, p.y * fdot + w.y * gdot, p.z * fdot + w.z * gdot);
    p = p1;
    w = w1;
    return true;
}

// drift_one: the drift, else ten substeps of dt/10 (stopping at a failed one).
// The flag is discarded by all MVS/HYBRID callers (mdt_mvs, mdt_hy, mco_mvs2h).
// Written as one loop so that drift_dan is instantiated once: attempt 0 is the
// whole step, attempts 1..10 the substeps.
__device__ __forceinline__ void drift_one(double mu, double3& p, double3& w, double dt) {
    const double sub = dt / 10.0;
#pragma unroll 1
    for (int attempt = 0; attempt <= 10; ++attempt) {
        const bool ok = drift_dan(mu, p, w, attempt == 0 ? dt : sub);
        if (attempt == 0 ? ok : !ok) return;
    }
}

}  // namespace mb200
