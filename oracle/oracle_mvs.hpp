// Test infrastructure only: CPU restatement of MERCURY6's mixed-variable
// symplectic (MVS) test-particle path, statement for statement, so that its
// results round exactly as the reference CPU build (mercury6_2.for compiled
// with -ffp-contract=off) does. Never linked into the product library.
//
// Index convention: C index k is Fortran body k+1; index 0 is the central body,
// 1..nbig-1 are the Big bodies, nbig..nbod-1 the Small bodies. Positions and
// velocities keep the Fortran layout x(3,nbod): x[3*k+c].
#pragma once
#include <vector>
#include "oracle_scalar.hpp"

namespace oracle {

// Constants of mercury.inc / swift.inc.
constexpr double K2 = 2.959122082855911e-4;
constexpr double HUGE_ = 9.9e29;
constexpr double PI = 3.141592653589793;
constexpr double TWOPI_SWIFT = 2.0 * PI;  // swift.inc: TWOPI = 2.0D0 * PI
constexpr double DANBYB = 1.0e-13;        // swift.inc convergence criterion

// Event record with the layout of the reference C ABI's MercuryEvent
// (mercury_cuda.h:7-11): 1-based ids, kind bits 1 close encounter,
// 2 near miss, 4 collision, 8 central impact.
struct Event {
    int i, j, kind, now;
    double distance, time;
    double xi[6], xj[6];
};

// ---------------------------------------------------------------- Kepler drift
// mco_sine, mercury6_2.for:2940-2972.
template <class R> void mco_sine(R& x, R& sx, R& cx) {
    const R pi = 3.141592653589793;
    const R twopi = R(2.0) * pi;
    if (x > R(0.0)) x = Fmod(x, twopi);
    else x = Fmod(x, twopi) + twopi;
    cx = Cos(x);
    if (x > pi) sx = -Sqrt(R(1.0) - cx * cx);
    else sx = Sqrt(R(1.0) - cx * cx);
}

// drift_kepu_stumpff, mercury6_2.for:8213-8266. Stumpff functions c0..c3 of x
// by argument quartering, the degree-6 series (coefficients (-1)^k/(2k+2)! and
// (-1)^k/(2k+3)! written as the Fortran literals), then the doubling recurrences.
template <class R> void drift_kepu_stumpff(R& x, R& c0, R& c1, R& c2, R& c3) {
    int n = 0;
    const R xm = 0.1;
    // Finite arguments fall below xm within ~520 passes; the cap (absent in
    // the Fortran) only keeps a non-finite argument from looping forever.
    while (Fabs(x) >= xm && n < 2000) {
        n = n + 1;
        x = x * R(0.25);
    }
    R x2 = x * x, x3 = x * x2, x4 = x2 * x2, x5 = x2 * x3, x6 = x3 * x3;
    c2 = R(1.147074559772972e-11) * x6 - R(2.087675698786810e-9) * x5 +
         R(2.755731922398589e-7) * x4 - R(2.480158730158730e-5) * x3 +
         R(1.388888888888889e-3) * x2 - R(4.166666666666667e-2) * x + R(0.5);
    c3 = R(7.647163731819816e-13) * x6 - R(1.605904383682161e-10) * x5 +
         R(2.505210838544172e-8) * x4 - R(2.755731922398589e-6) * x3 +
         R(1.984126984126984e-4) * x2 - R(8.333333333333333e-3) * x +
         R(1.666666666666667e-1);
    c1 = R(1.0) - x * c3;
    c0 = R(1.0) - x * c2;
    for (int i = n; i >= 1; --i) {
        c3 = (c2 + c0 * c3) * R(0.25);
        c2 = c1 * c1 * R(0.5);
        c1 = c0 * c1;
        c0 = R(2.0) * c0 * c0 - R(1.0);
        x = x * R(4.0);
    }
}

// drift_kepu_fchk, mercury6_2.for:7860-7882.
template <class R> void drift_kepu_fchk(R dt, R r0, R mu, R alpha, R u, R s, R& f) {
    R x = s * s * alpha, c0, c1, c2, c3;
    drift_kepu_stumpff(x, c0, c1, c2, c3);
    c1 = c1 * s;
    c2 = c2 * s * s;
    c3 = c3 * s * s * s;
    f = r0 * c1 + u * c2 + mu * c3 - dt;
}

// drift_kepu_p3solve, mercury6_2.for:8147-8194 (cubic seed for alpha <= 0).
template <class R> void drift_kepu_p3solve(R dt, R r0, R mu, R alpha, R u, R& s, int& iflg) {
    R denom = (mu - alpha * r0) / R(6.0);
    R a2 = R(0.5) * u / denom;
    R a1 = r0 / denom;
    R a0 = -dt / denom;
    R q = (a1 - a2 * a2 / R(3.0)) / R(3.0);
    R r = (a1 * a2 - R(3.0) * a0) / R(6.0) - Pow(a2, R(3.0)) / R(27.0);
    R sq2 = Pow(q, R(3.0)) + r * r;
    if (sq2 >= R(0.0)) {
        R sq = Sqrt(sq2), p1, p2;
        const R third = R(1.0) / R(3.0);
        if ((r + sq) <= R(0.0)) p1 = -Pow(-(r + sq), third);
        else p1 = Pow(r + sq, third);
        if ((r - sq) <= R(0.0)) p2 = -Pow(-(r - sq), third);
        else p2 = Pow(r - sq, third);
        iflg = 0;
        s = p1 + p2 - a2 / R(3.0);
    } else {
        iflg = 1;
        s = R(0.0);
    }
}

// drift_kepu_guess, mercury6_2.for:7906-7955.
template <class R> void drift_kepu_guess(R dt, R r0, R mu, R alpha, R u, R& s) {
    if (alpha > R(0.0)) {
        if (dt / r0 <= R(0.4)) {
            s = dt / r0 - (dt * dt * u) / (R(2.0) * r0 * r0 * r0);
            return;
        }
        R a = mu / alpha;
        R en = Sqrt(mu / (a * a * a));
        R ec = R(1.0) - r0 / a;
        R es = u / (en * a * a);
        R e = Sqrt(ec * ec + es * es);
        R y = en * dt - es, sy, cy;
        mco_sine(y, sy, cy);
        R sigma = Sign(R(1.0), es * cy + ec * sy);
        R x = y + sigma * R(0.85) * e;
        s = x / Sqrt(alpha);
    } else {
        int iflg;
        drift_kepu_p3solve(dt, r0, mu, alpha, u, s, iflg);
        if (iflg != 0) s = dt / r0;
    }
}

// The tangent of the universal-variable solve. Both solvers below stop once
// the residual at the current anomaly s_k is below DANBYB and return the
// Stumpff terms at s_k. Their values are converged, but the derivative that
// flows through the iterations is that of the iterate before the last one
// and can be far from the root's own derivative when the iteration started
// from a poor guess: a perturbation of 1e-10 already changes the number of
// iterations, and finite differences of the map see the root's derivative
// ds/dtheta = -F_theta / F_s. kepu_tangent replaces the tangent of s_k by
// that one (one Newton update of the tangent alone) and recomputes the
// returned terms from it; the values stay what they were. A no-op for plain
// and counting scalars; the dual-number overload is beside Dual.
template <class R>
inline void kepu_tangent(R&, const R&, const R&, const R&, const R&, const R&, R&, R&, R&, R&) {}

// drift_kepu_new, mercury6_2.for:8073-8122: up to 7 quartic Newton iterations.
template <class R>
void drift_kepu_new(R& s, R dt, R r0, R mu, R alpha, R u, R& fp, R& c1, R& c2, R& c3, int& iflgn) {
    for (int nc = 0; nc <= 6; ++nc) {
        R sk = s;
        R s2 = s * s;
        R x = s2 * alpha, c0;
        drift_kepu_stumpff(x, c0, c1, c2, c3);
        c1 = c1 * s;
        c2 = c2 * s2;
        c3 = c3 * s * s2;
        R f = r0 * c1 + u * c2 + mu * c3 - dt;
        fp = r0 * c0 + u * c1 + mu * c2;
        R fpp = (mu - r0 * alpha) * c1 + u * c0;
        R fppp = (mu - r0 * alpha) * c0 - u * alpha * c1;
        R ds = -(f / fp);
        ds = -(f / (fp + R(0.5) * ds * fpp));
        ds = -(f / (fp + R(0.5) * ds * fpp + ds * ds * fppp * R(0.1666666666666667)));
        s = s + ds;
        R fdt = f / dt;
        if (fdt * fdt < R(DANBYB) * R(DANBYB)) {
            iflgn = 0;
            kepu_tangent(sk, dt, r0, mu, alpha, u, fp, c1, c2, c3);
            return;
        }
    }
    iflgn = 1;
}

// drift_kepu_lag, mercury6_2.for:7984-8043: Laguerre fallback, at most 401 passes.
template <class R>
void drift_kepu_lag(R& s, R dt, R r0, R mu, R alpha, R u, R& fp, R& c1, R& c2, R& c3, int& iflg) {
    const int ncmax = 400;
    const R ln = 5.0;
    for (int nc = 0; nc <= ncmax; ++nc) {
        R sk = s;
        R x = s * s * alpha, c0;
        drift_kepu_stumpff(x, c0, c1, c2, c3);
        c1 = c1 * s;
        c2 = c2 * s * s;
        c3 = c3 * s * s * s;
        R f = r0 * c1 + u * c2 + mu * c3 - dt;
        fp = r0 * c0 + u * c1 + mu * c2;
        R fpp = (R(-40.0) * alpha + mu) * c1 + u * c0;
        R ds = -(ln * f / (fp + Sign(R(1.0), fp) *
                                   Sqrt(Fabs((ln - R(1.0)) * (ln - R(1.0)) * fp * fp -
                                             (ln - R(1.0)) * ln * f * fpp))));
        s = s + ds;
        R fdt = f / dt;
        if (fdt * fdt < R(DANBYB) * R(DANBYB)) {
            iflg = 0;
            kepu_tangent(sk, dt, r0, mu, alpha, u, fp, c1, c2, c3);
            return;
        }
    }
    iflg = 2;
}

// drift_kepu, mercury6_2.for:7802-7836.
template <class R>
void drift_kepu(R dt, R r0, R mu, R alpha, R u, R& fp, R& c1, R& c2, R& c3, int& iflg) {
    R s, fo, fn;
    drift_kepu_guess(dt, r0, mu, alpha, u, s);
    R st = s;
    drift_kepu_new(s, dt, r0, mu, alpha, u, fp, c1, c2, c3, iflg);
    if (iflg != 0) {
        drift_kepu_fchk(dt, r0, mu, alpha, u, st, fo);
        drift_kepu_fchk(dt, r0, mu, alpha, u, s, fn);
        if (Fabs(fo) < Fabs(fn)) s = st;
        drift_kepu_lag(s, dt, r0, mu, alpha, u, fp, c1, c2, c3, iflg);
    }
}

// drift_kepmd, mercury6_2.for:7730-7776: elliptic small-dm solver.
template <class R> void drift_kepmd(R dm, R es, R ec, R& x, R& s, R& c) {
    const R A0 = 39916800.0, A1 = 6652800.0, A2 = 332640.0, A3 = 7920.0, A4 = 110.0;
    R fac1 = R(1.0) / (R(1.0) - ec);
    R q = fac1 * dm;
    R fac2 = es * es * fac1 - ec / R(3.0);
    x = q * (R(1.0) - R(0.5) * fac1 * q * (es - q * fac2));
    R y = x * x;
    s = x * (A0 - y * (A1 - y * (A2 - y * (A3 - y * (A4 - y))))) / A0;
    c = Sqrt(R(1.0) - s * s);
    R f = x - ec * s + es * (R(1.0) - c) - dm;
    R fp = R(1.0) - ec * c + es * s;
    R fpp = ec * s + es * c;
    R fppp = ec * c - es * s;
    R dx = -(f / fp);
    dx = -(f / (fp + R(0.5) * dx * fpp));
    dx = -(f / (fp + R(0.5) * dx * fpp + R(0.16666666666666666) * dx * dx * fppp));
    x = x + dx;
    y = x * x;
    s = x * (A0 - y * (A1 - y * (A2 - y * (A3 - y * (A4 - y))))) / A0;
    c = Sqrt(R(1.0) - s * s);
}

// drift_dan, mercury6_2.for:7602-7709. Updates (x0..vz0) in place.
template <class R>
void drift_dan(R mu, R& x0, R& y0, R& z0, R& vx0, R& vy0, R& vz0, R dt0, int& iflg) {
    R dt = dt0;
    iflg = 0;
    R r0 = Sqrt(x0 * x0 + y0 * y0 + z0 * z0);
    R v0s = vx0 * vx0 + vy0 * vy0 + vz0 * vz0;
    R u = x0 * vx0 + y0 * vy0 + z0 * vz0;
    R alpha = R(2.0) * mu / r0 - v0s;
    R fp, c1, c2, c3;
    if (alpha > R(0.0)) {
        R a = mu / alpha;
        R asq = a * a;
        R en = Sqrt(mu / (a * asq));
        R ec = R(1.0) - r0 / a;
        R es = u / (en * asq);
        R esq = ec * ec + es * es;
        R dm = dt * en - R(double(int(val(dt * en / R(TWOPI_SWIFT))))) * R(TWOPI_SWIFT);
        dt = dm / en;
        if (!((dm * dm > R(0.16)) || (esq > R(0.36)))) {
            if (esq * dm * dm < R(0.0016)) {
                R xkep, s, c;
                drift_kepmd(dm, es, ec, xkep, s, c);
                R fchk = (xkep - ec * s + es * (R(1.0) - c) - dm);
                if (fchk * fchk > R(DANBYB)) {
                    iflg = 1;
                    return;
                }
                fp = R(1.0) - ec * c + es * s;
                R f = (a / r0) * (c - R(1.0)) + R(1.0);
                R g = dt + (s - xkep) / en;
                R fdot = -(a / (r0 * fp)) * en * s;
                R gdot = (c - R(1.0)) / fp + R(1.0);
                R x = x0 * f + vx0 * g, y = y0 * f + vy0 * g, z = z0 * f + vz0 * g;
                R vx = x0 * fdot + vx0 * gdot, vy = y0 * fdot + vy0 * gdot,
                  vz = z0 * fdot + vz0 * gdot;
                x0 = x; y0 = y; z0 = z;
                vx0 = vx; vy0 = vy; vz0 = vz;
                iflg = 0;
                return;
            }
        }
    }
    drift_kepu(dt, r0, mu, alpha, u, fp, c1, c2, c3, iflg);
    if (iflg == 0) {
        R f = R(1.0) - (mu / r0) * c2;
        R g = dt - mu * c3;
        R fdot = -(mu / (fp * r0)) * c1;
        R gdot = R(1.0) - (mu / fp) * c2;
        R x = x0 * f + vx0 * g, y = y0 * f + vy0 * g, z = z0 * f + vz0 * g;
        R vx = x0 * fdot + vx0 * gdot, vy = y0 * fdot + vy0 * gdot, vz = z0 * fdot + vz0 * gdot;
        x0 = x; y0 = y; z0 = z;
        vx0 = vx; vy0 = vy; vz0 = vz;
    }
}

// drift_one, mercury6_2.for:8296-8330: one drift, else ten substeps of dt/10
// (a failed substep leaves the partial result, which every caller keeps).
template <class R>
void drift_one(R mu, R& x, R& y, R& z, R& vx, R& vy, R& vz, R dt, int& iflg) {
    drift_dan(mu, x, y, z, vx, vy, vz, dt, iflg);
    if (iflg != 0) {
        for (int i = 1; i <= 10; ++i) {
            R dttmp = dt / R(10.0);
            drift_dan(mu, x, y, z, vx, vy, vz, dttmp, iflg);
            if (iflg != 0) return;
        }
    }
}

// ---------------------------------------------------------- coordinate maps
// mco_h2j, mercury6_2.for:2613-2682 (Big bodies only; Small bodies' Jacobi
// coordinates equal their heliocentric ones).
template <class R> void mco_h2j(int nbig, const R* m, const R* xh, const R* vh, R* x, R* v) {
    if (nbig < 2) return;
    R mtot = m[1];
    for (int c = 0; c < 3; ++c) { x[3 + c] = xh[3 + c]; v[3 + c] = vh[3 + c]; }
    R mx[3], mv[3];
    for (int c = 0; c < 3; ++c) { mx[c] = m[1] * xh[3 + c]; mv[c] = m[1] * vh[3 + c]; }
    for (int j = 2; j <= nbig - 2; ++j) {
        R temp = R(1.0) / (mtot + m[0]);
        mtot = mtot + m[j];
        for (int c = 0; c < 3; ++c) {
            x[3 * j + c] = xh[3 * j + c] - temp * mx[c];
            v[3 * j + c] = vh[3 * j + c] - temp * mv[c];
        }
        for (int c = 0; c < 3; ++c) {
            mx[c] = mx[c] + m[j] * xh[3 * j + c];
            mv[c] = mv[c] + m[j] * vh[3 * j + c];
        }
    }
    if (nbig > 2) {
        R temp = R(1.0) / (mtot + m[0]);
        int j = nbig - 1;
        for (int c = 0; c < 3; ++c) {
            x[3 * j + c] = xh[3 * j + c] - temp * mx[c];
            v[3 * j + c] = vh[3 * j + c] - temp * mv[c];
        }
    }
}

// mco_j2h, mercury6_2.for:2700-2770 (Big bodies only).
template <class R> void mco_j2h(int nbig, const R* m, const R* x, const R* v, R* xh, R* vh) {
    if (nbig < 2) return;
    for (int c = 0; c < 3; ++c) { xh[3 + c] = x[3 + c]; vh[3 + c] = v[3 + c]; }
    R mtot = m[1];
    R temp = m[1] / (mtot + m[0]);
    R mx[3], mv[3];
    for (int c = 0; c < 3; ++c) { mx[c] = temp * x[3 + c]; mv[c] = temp * v[3 + c]; }
    for (int j = 2; j <= nbig - 2; ++j) {
        for (int c = 0; c < 3; ++c) {
            xh[3 * j + c] = x[3 * j + c] + mx[c];
            vh[3 * j + c] = v[3 * j + c] + mv[c];
        }
        mtot = mtot + m[j];
        temp = m[j] / (mtot + m[0]);
        for (int c = 0; c < 3; ++c) {
            mx[c] = mx[c] + temp * x[3 * j + c];
            mv[c] = mv[c] + temp * v[3 * j + c];
        }
    }
    if (nbig > 2) {
        int j = nbig - 1;
        for (int c = 0; c < 3; ++c) {
            xh[3 * j + c] = x[3 * j + c] + mx[c];
            vh[3 * j + c] = v[3 * j + c] + mv[c];
        }
    }
}

// ------------------------------------------------------------------ forces
// mfo_obl, mercury6_2.for:5176-5230. jcen = J2 R^2, J4 R^4, J6 R^6.
template <class R>
void mfo_obl(const double* jcen, int nbod, const R* m, const R* x, R* a, R* acen) {
    acen[0] = 0.0; acen[1] = 0.0; acen[2] = 0.0;
    for (int i = 1; i < nbod; ++i) {
        const R* p = x + 3 * i;
        R r2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
        R r_1 = R(1.0) / Sqrt(r2);
        R r_2 = r_1 * r_1;
        R r_3 = r_2 * r_1;
        R jr2 = R(jcen[0]) * r_2;
        R jr4 = R(jcen[1]) * r_2 * r_2;
        R jr6 = R(jcen[2]) * r_2 * r_2 * r_2;
        R u2 = p[2] * p[2] * r_2;
        R u4 = u2 * u2;
        R u6 = u4 * u2;
        R tmp1 = m[0] * r_3;
        R tmp2 = jr2 * (R(7.5) * u2 - R(1.5)) +
                 jr4 * (R(39.375) * u4 - R(26.25) * u2 + R(1.875)) +
                 jr6 * (R(187.6875) * u6 - R(216.5625) * u4 + R(59.0625) * u2 - R(2.1875));
        R tmp3 = jr2 * R(3.0) + jr4 * (R(17.5) * u2 - R(7.5)) +
                 jr6 * (R(86.625) * u4 - R(78.75) * u2 + R(13.125));
        a[3 * i + 0] = p[0] * tmp1 * tmp2;
        a[3 * i + 1] = p[1] * tmp1 * tmp2;
        a[3 * i + 2] = p[2] * tmp1 * (tmp2 - tmp3);
        R tmp4 = m[i] / m[0];
        acen[0] = acen[0] - tmp4 * a[3 * i + 0];
        acen[1] = acen[1] - tmp4 * a[3 * i + 1];
        acen[2] = acen[2] - tmp4 * a[3 * i + 2];
    }
}

// mfo_ngf, mercury6_2.for:5106-5153: Marsden A1/A2/A3 (with the 88 AU^2
// cutoff) and the inverse-square transverse Yarkovsky term yar. ngf(5,nbod).
// Returns nonzero where the Fortran calls fail().
template <class R> int mfo_ngf(int nbod, const R* x, const R* v, R* a, const R* ngf) {
    for (int k = 0; k < 3 * nbod; ++k) a[k] = 0.0;
    for (int j = 1; j < nbod; ++j) {
        const R* g5 = ngf + 5 * j;
        const R* p = x + 3 * j;
        const R* u = v + 3 * j;
        if (g5[0] == R(0.0) && g5[1] == R(0.0) && g5[2] == R(0.0) && g5[4] == R(0.0)) continue;
        R r2 = R(0.0) + p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
        R r = Sqrt(r2);
        R rv = (R(0.0) + p[0] * u[0] + p[1] * u[1] + p[2] * u[2]) / r2;
        R tx = u[0] - rv * p[0], ty = u[1] - rv * p[1], tz = u[2] - rv * p[2];
        R tn = Sqrt(tx * tx + ty * ty + tz * tz);
        bool any = g5[0] != R(0.0) || g5[1] != R(0.0) || g5[2] != R(0.0);
        bool big = Fabs(g5[0]) > R(1e-7) || Fabs(g5[1]) > R(1e-7) || Fabs(g5[2]) > R(1e-7);
        R* aj = a + 3 * j;
        if (any && (r2 < R(88.0) || big)) {
            R q = r * R(0.3561253561253561);
            R g = R(0.111262) * Pow(q, R(-2.15)) * Pow(R(1.0) + Pow(q, R(5.093)), R(-4.6142));
            for (int c = 0; c < 3; ++c) aj[c] = g5[0] * g / r * p[c];
            if (g5[1] != R(0.0)) {
                if (tn == R(0.0)) return 1;
                R f = g5[1] * g / tn;
                aj[0] = aj[0] + f * tx; aj[1] = aj[1] + f * ty; aj[2] = aj[2] + f * tz;
            }
            if (g5[2] != R(0.0)) {
                R nx = p[1] * u[2] - p[2] * u[1];
                R ny = p[2] * u[0] - p[0] * u[2];
                R nz = p[0] * u[1] - p[1] * u[0];
                R nn = Sqrt(nx * nx + ny * ny + nz * nz);
                if (nn == R(0.0)) return 1;
                R f = g5[2] * g / nn;
                aj[0] = aj[0] + f * nx; aj[1] = aj[1] + f * ny; aj[2] = aj[2] + f * nz;
            }
        }
        if (g5[4] != R(0.0)) {
            if (tn == R(0.0)) return 1;
            R f = g5[4] / (r2 * tn);
            aj[0] = aj[0] + f * tx; aj[1] = aj[1] + f * ty; aj[2] = aj[2] + f * tz;
        }
    }
    return 0;
}

// mfo_mvs, mercury6_2.for:4929-5075: interaction-Hamiltonian accelerations of
// the MVS map. x heliocentric, xj Jacobi (Big bodies).
template <class R>
void mfo_mvs(const double* jcen, int nbod, int nbig, const R* m, const R* x, const R* xj, R* a) {
    if (nbod < 2) return;
    std::vector<R> a1(3 * nbig > 0 ? 3 * nbig : 1), a2(3 * nbig > 0 ? 3 * nbig : 1);
    std::vector<R> a3(3 * nbod);
    R a0[3] = {0.0, 0.0, 0.0};
    if (nbig >= 2) for (int c = 0; c < 3; ++c) { a1[3 + c] = 0.0; a2[3 + c] = 0.0; }
    R minside = 0.0;
    for (int k = 2; k < nbig; ++k) {
        int k1 = k - 1;
        minside = minside + m[k1];
        const R* p = x + 3 * k;
        const R* pj = xj + 3 * k;
        R r2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
        R rj2 = pj[0] * pj[0] + pj[1] * pj[1] + pj[2] * pj[2];
        R r = R(1.0) / Sqrt(r2);
        R rj = R(1.0) / Sqrt(rj2);
        R r3 = r * r * r;
        R rj3 = rj * rj * rj;
        R fac0 = m[k] * r3;
        R fac12 = m[0] * rj3;
        R fac2 = m[k] * fac12 / (minside + m[0]);
        R q = (r2 - rj2) * R(0.5) / rj2;
        R q2 = q * q, q3 = q * q2, q4 = q2 * q2, q5 = q2 * q3, q6 = q3 * q3, q7 = q3 * q4;
        R fac1 = R(402.1875) * q7 - R(187.6875) * q6 + R(86.625) * q5 - R(39.375) * q4 +
                 R(17.5) * q3 - R(7.5) * q2 + R(3.0) * q - R(1.0);
        for (int c = 0; c < 3; ++c) {
            a0[c] = a0[c] - fac0 * p[c];
            a1[3 * k + c] = fac12 * (pj[c] + fac1 * p[c]);
            a2[3 * k + c] = a2[3 * k1 + c] + fac2 * pj[c];
        }
    }
    R a0tp[3] = {0.0, 0.0, 0.0};
    if (nbig >= 2) {
        const R* p = x + 3;
        R r2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
        R r = R(1.0) / Sqrt(r2);
        R r3 = r * r * r;
        R fac0 = m[1] * r3;
        for (int c = 0; c < 3; ++c) a0tp[c] = a0[c] - fac0 * p[c];
    }
    for (int k = 1; k < nbod; ++k) for (int c = 0; c < 3; ++c) a3[3 * k + c] = 0.0;
    for (int i = 1; i < nbig; ++i) {
        for (int j = i + 1; j < nbig; ++j) {
            R dx = x[3 * j] - x[3 * i], dy = x[3 * j + 1] - x[3 * i + 1], dz = x[3 * j + 2] - x[3 * i + 2];
            R s2 = dx * dx + dy * dy + dz * dz;
            R s_1 = R(1.0) / Sqrt(s2);
            R s_3 = s_1 * s_1 * s_1;
            R faci = m[i] * s_3, facj = m[j] * s_3;
            a3[3 * j] = a3[3 * j] - faci * dx; a3[3 * j + 1] = a3[3 * j + 1] - faci * dy; a3[3 * j + 2] = a3[3 * j + 2] - faci * dz;
            a3[3 * i] = a3[3 * i] + facj * dx; a3[3 * i + 1] = a3[3 * i + 1] + facj * dy; a3[3 * i + 2] = a3[3 * i + 2] + facj * dz;
        }
        for (int j = nbig; j < nbod; ++j) {
            R dx = x[3 * j] - x[3 * i], dy = x[3 * j + 1] - x[3 * i + 1], dz = x[3 * j + 2] - x[3 * i + 2];
            R s2 = dx * dx + dy * dy + dz * dz;
            R s_1 = R(1.0) / Sqrt(s2);
            R s_3 = s_1 * s_1 * s_1;
            R faci = m[i] * s_3;
            a3[3 * j] = a3[3 * j] - faci * dx; a3[3 * j + 1] = a3[3 * j + 1] - faci * dy; a3[3 * j + 2] = a3[3 * j + 2] - faci * dz;
        }
    }
    for (int k = 1; k < nbig; ++k)
        for (int c = 0; c < 3; ++c) a[3 * k + c] = a0[c] + a1[3 * k + c] + a2[3 * k + c] + a3[3 * k + c];
    for (int k = nbig; k < nbod; ++k)
        for (int c = 0; c < 3; ++c) a[3 * k + c] = a0tp[c] + a3[3 * k + c];
    if (jcen[0] != 0.0 || jcen[1] != 0.0 || jcen[2] != 0.0) {
        std::vector<R> aobl(3 * nbod);
        R acen[3];
        mfo_obl(jcen, nbod, m, x, aobl.data(), acen);
        for (int k = 1; k < nbod; ++k)
            for (int c = 0; c < 3; ++c) a[3 * k + c] = a[3 * k + c] + (aobl[3 * k + c] - acen[c]);
    }
}

// ------------------------------------------------------- encounter screens
// mce_box, mercury6_2.for:997-1040: x-y bounding boxes over the step.
template <class R>
void mce_box(int nbod, R h, const R* x0, const R* v0, const R* x1, const R* v1,
             R* xmin, R* xmax, R* ymin, R* ymax) {
    for (int j = 1; j < nbod; ++j) {
        R* lo[2] = {xmin + j, ymin + j};
        R* hi[2] = {xmax + j, ymax + j};
        for (int c = 0; c < 2; ++c) {
            R a0 = x0[3 * j + c], a1 = x1[3 * j + c], u0 = v0[3 * j + c], u1 = v1[3 * j + c];
            *lo[c] = Min(a0, a1);
            *hi[c] = Max(a0, a1);
            if ((u0 < R(0.0) && u1 > R(0.0)) || (u0 > R(0.0) && u1 < R(0.0))) {
                R temp = (u0 * a1 - u1 * a0 - R(0.5) * h * u0 * u1) / (u0 - u1);
                *lo[c] = Min(*lo[c], temp);
                *hi[c] = Max(*hi[c], temp);
            }
        }
    }
}

// mce_min, mercury6_2.for:1572-1622: cubic-interpolated minimum of d(t).
template <class R> void mce_min(R d0, R d1, R d0t, R d1t, R h, R& d2min, R& tmin) {
    if (d0t * h > R(0.0) || d1t * h < R(0.0)) {
        if (d0 <= d1) { d2min = d0; tmin = -h; }
        else { d2min = d1; tmin = 0.0; }
        return;
    }
    R temp = R(6.0) * (d0 - d1);
    R a = temp + R(3.0) * h * (d0t + d1t);
    R b = temp + R(2.0) * h * (d0t + R(2.0) * d1t);
    R c = h * d1t;
    temp = -(R(0.5) * (b + Sign(Sqrt(Max(b * b - R(4.0) * a * c, R(0.0))), b)));
    R tau;
    if (temp == R(0.0)) tau = 0.0;
    else tau = c / temp;
    tau = Min(tau, R(0.0));
    tau = Max(tau, R(-1.0));
    tmin = tau * h;
    temp = R(1.0) + tau;
    d2min = tau * tau * ((R(3.0) + R(2.0) * tau) * d0 + temp * h * d0t) +
            temp * temp * ((R(1.0) - R(2.0) * tau) * d1 + tau * h * d1t);
    d2min = Max(d2min, R(0.0));
}

// mce_stat, mercury6_2.for:1765-1918, emitting one record per qualifying pair
// in the reference ABI's merged form: kind bit 1 for a close-encounter minimum
// (the iclo/jclo list), bit 2 for a near miss and bit 4 for a collision (the
// ihit/jhit list with chit). time = tmin + time, xi/xj the linear
// interpolations of mce_stat:1869-1882. Body status flags are all taken as
// alive, as the GPU path assumes.
template <class R>
void mce_stat(R time, R h, int nbod, int nbig, const R* m, const R* x0, const R* v0,
              const R* x1, const R* v1, const R* rce, const R* rphys, std::vector<Event>& out) {
    R hm1 = R(1.0) / h;
    std::vector<R> xmin(nbod), xmax(nbod), ymin(nbod), ymax(nbod);
    mce_box(nbod, h, x0, v0, x1, v1, xmin.data(), xmax.data(), ymin.data(), ymax.data());
    for (int j = 1; j < nbod; ++j) {
        R temp = rce[j] * R(1.2);
        xmin[j] = xmin[j] - temp;
        xmax[j] = xmax[j] + temp;
        ymin[j] = ymin[j] - temp;
        ymax[j] = ymax[j] + temp;
    }
    for (int i = 1; i < nbig; ++i) {
        for (int j = i + 1; j < nbod; ++j) {
            if (!(xmax[i] >= xmin[j] && xmax[j] >= xmin[i] && ymax[i] >= ymin[j] && ymax[j] >= ymin[i]))
                continue;
            R dx0 = x0[3 * i] - x0[3 * j], dy0 = x0[3 * i + 1] - x0[3 * j + 1], dz0 = x0[3 * i + 2] - x0[3 * j + 2];
            R du0 = v0[3 * i] - v0[3 * j], dv0 = v0[3 * i + 1] - v0[3 * j + 1], dw0 = v0[3 * i + 2] - v0[3 * j + 2];
            R d0t = (dx0 * du0 + dy0 * dv0 + dz0 * dw0) * R(2.0);
            R dx1 = x1[3 * i] - x1[3 * j], dy1 = x1[3 * i + 1] - x1[3 * j + 1], dz1 = x1[3 * i + 2] - x1[3 * j + 2];
            R du1 = v1[3 * i] - v1[3 * j], dv1 = v1[3 * i + 1] - v1[3 * j + 1], dw1 = v1[3 * i + 2] - v1[3 * j + 2];
            R d1t = (dx1 * du1 + dy1 * dv1 + dz1 * dw1) * R(2.0);
            R d0 = dx0 * dx0 + dy0 * dy0 + dz0 * dz0;
            R d1 = dx1 * dx1 + dy1 * dy1 + dz1 * dz1;
            R d2min, tmin;
            mce_min(d0, d1, d0t, d1t, h, d2min, tmin);
            R d2ce = Max(rce[i], rce[j]);
            R d2hit = rphys[i] + rphys[j];
            d2ce = d2ce * d2ce;
            d2hit = d2hit * d2hit;
            R d2near = d2hit * R(4.0);
            bool clo = (d2min <= d2ce && d0t * h <= R(0.0) && d1t * h >= R(0.0)) || (d2min <= d2hit);
            bool near = d2min <= d2near;
            if (!clo && !near) continue;
            Event e{};
            int a = i, b = j;
            if (m[j] > m[i] && j < nbig) { a = j; b = i; }
            e.i = a + 1;
            e.j = b + 1;
            e.kind = (clo ? 1 : 0) | (near ? 2 : 0) | (d2min <= d2hit ? 4 : 0);
            e.now = d1 <= d2hit ? 1 : 0;
            e.time = val(tmin + time);
            e.distance = val(Sqrt(Max(R(0.0), d2min)));
            R tmp0 = -tmin * hm1;
            R tmp1 = R(1.0) + tmin * hm1;
            for (int c = 0; c < 3; ++c) {
                e.xi[c] = val(tmp0 * x0[3 * a + c] + tmp1 * x1[3 * a + c]);
                e.xi[c + 3] = val(tmp0 * v0[3 * a + c] + tmp1 * v1[3 * a + c]);
                e.xj[c] = val(tmp0 * x0[3 * b + c] + tmp1 * x1[3 * b + c]);
                e.xj[c + 3] = val(tmp0 * v0[3 * b + c] + tmp1 * v1[3 * b + c]);
            }
            out.push_back(e);
        }
    }
}

// mce_cent, mercury6_2.for:1059-1167 (algor != 11): pericentre passage within
// rcen of the central body over the step, with the entry time measured from
// the beginning of the signed step. Records have kind 8, i=1.
template <class R>
void mce_cent(R time, R h, R rcen, int i0, int nbod, const R* m, const R* x0, const R* v0,
              const R* x1, const R* v1, std::vector<Event>& out) {
    if (i0 <= 0) i0 = 1;
    R rcen2 = rcen * rcen;
    R mcen = m[0];
    for (int j = i0; j < nbod; ++j) {
        const R *p0 = x0 + 3 * j, *u0 = v0 + 3 * j, *p1 = x1 + 3 * j, *u1 = v1 + 3 * j;
        R rr0 = p0[0] * p0[0] + p0[1] * p0[1] + p0[2] * p0[2];
        R rr1 = p1[0] * p1[0] + p1[1] * p1[1] + p1[2] * p1[2];
        R rv0 = u0[0] * p0[0] + u0[1] * p0[1] + u0[2] * p0[2];
        R rv1 = u1[0] * p1[0] + u1[1] * p1[1] + u1[2] * p1[2];
        if (!((rv0 * h <= R(0.0) && rv1 * h >= R(0.0)) || Min(rr0, rr1) <= rcen2)) continue;
        R hx = p0[1] * u0[2] - p0[2] * u0[1];
        R hy = p0[2] * u0[0] - p0[0] * u0[2];
        R hz = p0[0] * u0[1] - p0[1] * u0[0];
        R v2 = u0[0] * u0[0] + u0[1] * u0[1] + u0[2] * u0[2];
        R h2 = hx * hx + hy * hy + hz * hz;
        R p = h2 / (mcen + m[j]);
        R r0 = Sqrt(rr0);
        R temp = R(1.0) + p * (v2 / (mcen + m[j]) - R(2.0) / r0);
        R e = Sqrt(Max(temp, R(0.0)));
        R q = p / (R(1.0) + e);
        if (!(q <= rcen)) continue;
        temp = 0.0;
        if (e > R(0.0) && e < R(1.0)) {
            R a = q / (R(1.0) - e);
            R uhit = Sign(Acos(Max(R(-1.0), Min(R(1.0), (R(1.0) - rcen / a) / e))), -h);
            R uu0 = Sign(Acos(Max(R(-1.0), Min(R(1.0), (R(1.0) - r0 / a) / e))), rv0);
            R mhit = uhit - e * Sin(uhit);
            R m0 = uu0 - e * Sin(uu0);
            temp = (mhit - m0) / Sqrt((mcen + m[j]) / (a * a * a));
        } else if (e > R(1.0)) {
            R a = q / (e - R(1.0));
            R uhit = Sign(Acosh(Max(R(1.0), (R(1.0) + rcen / a) / e)), -h);
            R uu0 = Sign(Acosh(Max(R(1.0), (R(1.0) + r0 / a) / e)), rv0);
            R mhit = e * Sinh(uhit) - uhit;
            R m0 = e * Sinh(uu0) - uu0;
            temp = (mhit - m0) / Sqrt((mcen + m[j]) / (a * a * a));
        } else if (e == R(1.0) && q > R(0.0)) {
            R uhit = Sign(Sqrt(Max(R(0.0), rcen / q - R(1.0))), -h);
            R uu0 = Sign(Sqrt(Max(R(0.0), r0 / q - R(1.0))), rv0);
            // Integer powers q**3 expand to (q*q)*q, as gfortran's powi does.
            temp = Sqrt(R(2.0) * (q * q * q) / (mcen + m[j])) *
                   (uhit + (uhit * uhit * uhit) / R(3.0) - uu0 - (uu0 * uu0 * uu0) / R(3.0));
        }
        if (q == R(0.0) && rr1 != rr0)
            temp = h * Max(R(0.0), Min(R(1.0), (r0 - rcen) / (r0 - Sqrt(rr1))));
        Event ev{};
        ev.i = 1;
        ev.j = j + 1;
        ev.kind = 8;
        ev.time = val(time - h + temp);
        ev.distance = val(rcen);
        out.push_back(ev);
    }
}

// ------------------------------------------------------------- MVS step
// Persistent state of mdt_mvs between calls (its Fortran SAVE variables) plus
// the dtflag handshake of mal_hcon: dtflag != 2 recomputes the cached
// accelerations before the first kick.
template <class R> struct MvsState {
    std::vector<R> a, angf, xj, vj, gm, x0, v0;
    int dtflag = 0;
    void size(int nbod) {
        if ((int)a.size() < 3 * nbod) {
            a.assign(3 * nbod, R(0.0));
            angf.assign(3 * nbod, R(0.0));
            xj.assign(3 * nbod, R(0.0));
            vj.assign(3 * nbod, R(0.0));
            gm.assign(nbod, R(0.0));
            x0.assign(3 * nbod, R(0.0));
            v0.assign(3 * nbod, R(0.0));
        }
    }
};

// mdt_mvs, mercury6_2.for:3987-4101. ngf holds five coefficients per body.
// The user-force hook (ausr) is zero: the CUDA path rejects mfo_user.
template <class R>
int mdt_mvs(R time, R h0, const double* jcen, int nbod, int nbig, const R* m, R* x, R* v,
            const R* rce, const R* rphys, const R* ngf, int ngflag, MvsState<R>& st,
            std::vector<Event>& events) {
    st.size(nbod);
    R hby2 = R(0.5) * h0;
    const R ausr = 0.0;
    if (st.dtflag != 2) {
        st.dtflag = 2;
        mco_h2j(nbig, m, x, v, st.xj.data(), st.vj.data());
        mfo_mvs(jcen, nbod, nbig, m, x, st.xj.data(), st.a.data());
        R minside = m[0];
        for (int j = 1; j < nbig; ++j) {
            R msofar = minside + m[j];
            st.gm[j] = m[0] * msofar / minside;
            minside = msofar;
            for (int c = 0; c < 3; ++c) st.angf[3 * j + c] = 0.0;
        }
        if (ngflag == 1 || ngflag == 3)
            if (mfo_ngf(nbod, x, v, st.angf.data(), ngf)) return 1;
    }
    for (int j = 1; j < nbod; ++j)
        for (int c = 0; c < 3; ++c)
            v[3 * j + c] = v[3 * j + c] + hby2 * (st.angf[3 * j + c] + ausr + st.a[3 * j + c]);
    for (int k = 0; k < 3 * nbod; ++k) { st.x0[k] = x[k]; st.v0[k] = v[k]; }
    mco_h2j(nbig, m, x, v, st.xj.data(), st.vj.data());
    int iflag;
    for (int j = 1; j < nbig; ++j) {
        iflag = 0;
        R* q = st.xj.data() + 3 * j;
        R* w = st.vj.data() + 3 * j;
        drift_one(st.gm[j], q[0], q[1], q[2], w[0], w[1], w[2], h0, iflag);
    }
    for (int j = nbig; j < nbod; ++j) {
        iflag = 0;
        R* q = x + 3 * j;
        R* w = v + 3 * j;
        drift_one(m[0], q[0], q[1], q[2], w[0], w[1], w[2], h0, iflag);
    }
    mco_j2h(nbig, m, st.xj.data(), st.vj.data(), x, v);
    R temp = time + h0;
    mce_stat(temp, h0, nbod, nbig, m, st.x0.data(), st.v0.data(), x, v, rce, rphys, events);
    mfo_mvs(jcen, nbod, nbig, m, x, st.xj.data(), st.a.data());
    if (ngflag == 1 || ngflag == 3)
        if (mfo_ngf(nbod, x, v, st.angf.data(), ngf)) return 1;
    for (int j = 1; j < nbod; ++j)
        for (int c = 0; c < 3; ++c)
            v[3 * j + c] = v[3 * j + c] + hby2 * (st.angf[3 * j + c] + ausr + st.a[3 * j + c]);
    return 0;
}

// mco_mvs2h (forward=true, mercury6_2.for:2107-2227) and mco_h2mvs
// (forward=false, mercury6_2.for:2420-2535): the two-stage symplectic
// corrector between MVS map variables and heliocentric coordinates.
template <class R>
int mvs_corrector(bool forward, R h, const double* jcen, int nbod, int nbig, const R* m,
                  const R* x, const R* v, const R* ngf, int ngflag, R* xh, R* vh) {
    R rt10 = Sqrt(R(10.0));
    R ha[2], hb[2];
    if (forward) {
        ha[0] = h * rt10 * R(3.0) / R(10.0);
        hb[0] = -(h * rt10 / R(72.0));
        ha[1] = h * rt10 / R(5.0);
        hb[1] = h * rt10 / R(24.0);
    } else {
        ha[0] = -(h * rt10 / R(5.0));
        hb[0] = -(h * rt10 / R(24.0));
        ha[1] = -(h * rt10 * R(3.0) / R(10.0));
        hb[1] = h * rt10 / R(72.0);
    }
    std::vector<R> gm(nbod), a(3 * nbod), xj(3 * nbod), vj(3 * nbod), angf(3 * nbod, R(0.0));
    const R ausr = 0.0;
    for (int k = 0; k < 3 * nbod; ++k) { xh[k] = x[k]; vh[k] = v[k]; }
    R minside = m[0];
    for (int j = 1; j < nbig; ++j) {
        R msofar = minside + m[j];
        gm[j] = m[0] * msofar / minside;
        minside = msofar;
    }
    auto drift_all = [&](R dt) {
        mco_h2j(nbig, m, xh, vh, xj.data(), vj.data());
        int iflag;
        for (int j = 1; j < nbig; ++j) {
            iflag = 0;
            drift_one(gm[j], xj[3 * j], xj[3 * j + 1], xj[3 * j + 2], vj[3 * j], vj[3 * j + 1], vj[3 * j + 2], dt, iflag);
        }
        for (int j = nbig; j < nbod; ++j) {
            iflag = 0;
            drift_one(m[0], xh[3 * j], xh[3 * j + 1], xh[3 * j + 2], vh[3 * j], vh[3 * j + 1], vh[3 * j + 2], dt, iflag);
        }
        mco_j2h(nbig, m, xj.data(), vj.data(), xh, vh);
    };
    auto kick = [&](R hk, bool subtract) -> int {
        mfo_mvs(jcen, nbod, nbig, m, xh, xj.data(), a.data());
        if (ngflag == 1 || ngflag == 3)
            if (mfo_ngf(nbod, xh, vh, angf.data(), ngf)) return 1;
        for (int j = 1; j < nbod; ++j)
            for (int c = 0; c < 3; ++c) {
                R term = hk * (angf[3 * j + c] + ausr + a[3 * j + c]);
                vh[3 * j + c] = subtract ? vh[3 * j + c] - term : vh[3 * j + c] + term;
            }
        return 0;
    };
    for (int k = 0; k < 2; ++k) {
        drift_all(ha[k]);
        if (kick(hb[k], forward)) return 1;
        drift_all(R(-2.0) * ha[k]);
        if (kick(hb[k], !forward)) return 1;
        drift_all(ha[k]);
    }
    return 0;
}

// mce_hill, mercury6_2.for:1285-1314 with mco_x2a, mercury6_2.for:3013-3035.
template <class R> void mce_hill(int nbod, const R* m, const R* x, const R* v, R* hill, R* a) {
    const R THIRD = 0.3333333333333333;
    for (int j = 1; j < nbod; ++j) {
        R gm = m[0] + m[j];
        const R *p = x + 3 * j, *u = v + 3 * j;
        R r = Sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        R v2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        if (R(2.0) * gm == r * v2) a[j] = 0.0;
        else a[j] = gm * r / (R(2.0) * gm - r * v2);
        if (a[j] <= R(0.0)) a[j] = r;
        hill[j] = a[j] * Pow(THIRD * m[j] / m[0], THIRD);
    }
}

// mce_init's limits, mercury6_2.for:1339-1380 (the close-encounter file
// header it also writes is I/O and not restated): rce = hill * rceh,
// rphys = hill / a * (2.25 m1 / (pi rho))^(1/3), and with rcritflag
// rcrit = max(hill * cefac, 0.4 |h| sqrt(m1 / amin)).
template <class R>
void mce_init(R h, R cefac, int nbod, const R* m, const R* x, const R* v, const R* rho, const R* rceh, R* rphys,
              R* rce, R* rcrit, int rcritflag) {
    const R N2 = 0.4, THIRD = 0.3333333333333333, PI = 3.141592653589793;
    const R HUGE_ = 9.9e29;
    std::vector<R> a(nbod), hill(nbod);
    R amin = HUGE_;
    mce_hill(nbod, m, x, v, hill.data(), a.data());
    R temp = R(2.25) * m[0] / PI;
    for (int j = 1; j < nbod; ++j) {
        rce[j] = hill[j] * rceh[j];
        rphys[j] = hill[j] / a[j] * Pow(temp / rho[j], THIRD);
        amin = std::min(a[j], amin);
    }
    if (rcritflag == 1) {
        const R vmax = Sqrt(m[0] / amin);
        temp = N2 * std::fabs(h) * vmax;
        for (int j = 1; j < nbod; ++j) rcrit[j] = std::max(hill[j] * cefac, temp);
    }
}

}  // namespace oracle
