// Test infrastructure only: CPU restatement of MERCURY6's heliocentric force
// (mfo_all with mfo_grav's fused solar 1PN, mfo_obl, mfo_ngf, mfo_pr) and of
// the RA15 Gauss-Radau integrator (mdt_ra15), statement for statement.
#pragma once
#include <cmath>
#include <vector>

#include "oracle_mvs.hpp"

namespace oracle {

constexpr double AU_CM = 1.495978707e13;  // mercury.inc AU

// Speed of light in AU/day as mfo_grav/mfo_pr/mfo_pn compute it.
inline double light_speed() { return 299792458.0 * 86400.0 / (AU_CM * 0.01); }

// mfo_grav, mercury6_2.for:4593-4689 (pn != 0: the fused central-mass 1PN).
// Returns nonzero where the Fortran calls fail().
template <class R>
int mfo_grav(int nbod, int nbig, const R* m, const R* x, const R* v, R* a, int pn) {
    std::vector<R> r3(nbod), ri(nbod);
    R sx = 0.0, sy = 0.0, sz = 0.0;
    for (int i = 1; i < nbod; ++i) {
        a[3 * i] = 0.0; a[3 * i + 1] = 0.0; a[3 * i + 2] = 0.0;
        const R* p = x + 3 * i;
        R s2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
        if (s2 <= R(0.0)) return 1;
        R s_1 = R(1.0) / Sqrt(s2);
        ri[i] = s_1;
        r3[i] = s_1 * s_1 * s_1;
    }
    for (int i = 1; i < nbod; ++i) {
        R tmp1 = m[i] * r3[i];
        sx = sx - tmp1 * x[3 * i];
        sy = sy - tmp1 * x[3 * i + 1];
        sz = sz - tmp1 * x[3 * i + 2];
    }
    for (int i = 1; i < nbig; ++i) {
        for (int j = i + 1; j < nbod; ++j) {
            R dx = x[3 * j] - x[3 * i], dy = x[3 * j + 1] - x[3 * i + 1], dz = x[3 * j + 2] - x[3 * i + 2];
            R s2 = dx * dx + dy * dy + dz * dz;
            if (s2 <= R(0.0)) return 1;
            R s_1 = R(1.0) / Sqrt(s2);
            R s_3 = s_1 * s_1 * s_1;
            R tmp1 = s_3 * m[i];
            R tmp2 = s_3 * m[j];
            a[3 * j] = a[3 * j] - tmp1 * dx; a[3 * j + 1] = a[3 * j + 1] - tmp1 * dy; a[3 * j + 2] = a[3 * j + 2] - tmp1 * dz;
            a[3 * i] = a[3 * i] + tmp2 * dx; a[3 * i + 1] = a[3 * i + 1] + tmp2 * dy; a[3 * i + 2] = a[3 * i + 2] + tmp2 * dz;
        }
    }
    if (pn == 0) {
        for (int i = 1; i < nbod; ++i) {
            R tmp1 = m[0] * r3[i];
            a[3 * i] = a[3 * i] + sx - tmp1 * x[3 * i];
            a[3 * i + 1] = a[3 * i + 1] + sy - tmp1 * x[3 * i + 1];
            a[3 * i + 2] = a[3 * i + 2] + sz - tmp1 * x[3 * i + 2];
        }
    } else {
        const R c = R(light_speed());
        const R light2 = c * c;  // (...)**2 is an integer power: c*c
        for (int i = 1; i < nbod; ++i) {
            const R* p = x + 3 * i;
            const R* u = v + 3 * i;
            R tmp1 = m[0] * r3[i];
            R rv = R(0.0) + p[0] * u[0] + p[1] * u[1] + p[2] * u[2];
            R v2 = R(0.0) + u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
            R f = tmp1 / light2;
            R radial = R(4.0) * m[0] * ri[i] - v2;
            a[3 * i] = a[3 * i] + sx - tmp1 * p[0] + f * (radial * p[0] + R(4.0) * rv * u[0]);
            a[3 * i + 1] = a[3 * i + 1] + sy - tmp1 * p[1] + f * (radial * p[1] + R(4.0) * rv * u[1]);
            a[3 * i + 2] = a[3 * i + 2] + sz - tmp1 * p[2] + f * (radial * p[2] + R(4.0) * rv * u[2]);
        }
    }
    return 0;
}

// mfo_pr, mercury6_2.for:5307-5343: radiation pressure and Poynting-Robertson
// drag (solar-wind factor 0.3) for massless bodies with beta = ngf(4,j) != 0.
template <class R> void mfo_pr(int nbod, const R* m, const R* x, const R* v, R* a, const R* ngf) {
    const R c = R(light_speed());
    const R sw = 0.3;
    for (int j = 1; j < nbod; ++j) {
        R* aj = a + 3 * j;
        if (m[j] != R(0.0) || ngf[5 * j + 3] == R(0.0)) {
            aj[0] = 0.0; aj[1] = 0.0; aj[2] = 0.0;
            continue;
        }
        const R* p = x + 3 * j;
        const R* u = v + 3 * j;
        R r = Sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        R vr = (p[0] * u[0] + p[1] * u[1] + p[2] * u[2]) / r;
        R f = R(K2) * ngf[5 * j + 3] / (r * r);
        for (int k = 0; k < 3; ++k)
            aj[k] = f * ((R(1.0) - (R(1.0) + sw) * vr / c) * p[k] / r - (R(1.0) + sw) * u[k] / c);
    }
}

// mfo_pn, mercury6_2.for:5260-5279: the central-mass 1PN term alone.
template <class R> void mfo_pn(int nbod, const R* m, const R* x, const R* v, R* a) {
    const R c = R(light_speed());
    for (int k = 0; k < 3 * nbod; ++k) a[k] = 0.0;
    for (int j = 1; j < nbod; ++j) {
        const R* p = x + 3 * j;
        const R* u = v + 3 * j;
        R r2 = R(0.0) + p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
        R ri = R(1.0) / Sqrt(r2);
        R rv = R(0.0) + p[0] * u[0] + p[1] * u[1] + p[2] * u[2];
        R v2 = R(0.0) + u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        R f = m[0] * ri * ri * ri / (c * c);
        R radial = R(4.0) * m[0] * ri - v2;
        for (int k = 0; k < 3; ++k) a[3 * j + k] = f * (radial * p[k] + R(4.0) * rv * u[k]);
    }
}

// mfo_all, mercury6_2.for:4506-4571 (the user force is rejected by the CUDA
// path). Returns nonzero where a called routine would fail().
template <class R>
int mfo_all(const double* jcen, int nbod, int nbig, const R* m, const R* x, const R* v, R* a,
            const R* ngf, int ngflag, int pn) {
    if (mfo_grav(nbod, nbig, m, x, v, a, pn)) return 1;
    std::vector<R> acor(3 * nbod);
    if (jcen[0] != 0.0 || jcen[1] != 0.0 || jcen[2] != 0.0) {
        R acen[3];
        mfo_obl(jcen, nbod, m, x, acor.data(), acen);
        for (int j = 1; j < nbod; ++j)
            for (int k = 0; k < 3; ++k) a[3 * j + k] = a[3 * j + k] + (acor[3 * j + k] - acen[k]);
    }
    if (ngflag == 1 || ngflag == 3) {
        if (mfo_ngf(nbod, x, v, acor.data(), ngf)) return 1;
        for (int j = 1; j < nbod; ++j)
            for (int k = 0; k < 3; ++k) a[3 * j + k] = a[3 * j + k] + acor[3 * j + k];
    }
    if (ngflag == 2 || ngflag == 3) {
        mfo_pr(nbod, m, x, v, acor.data(), ngf);
        for (int j = 1; j < nbod; ++j)
            for (int k = 0; k < 3; ++k) a[3 * j + k] = a[3 * j + k] + acor[3 * j + k];
    }
    return 0;
}

// Constants of mdt_ra15 (mercury6_2.for:4164-4209): Gauss-Radau spacings h,
// series coefficients xc/vc and Everhart's r, c, d tables.
struct Ra15Constants {
    double h[8], xc[8], vc[7], r[28], c[21], d[21];
    Ra15Constants() {
        const double hh[8] = {0.0, .0562625605369221, .1802406917368924, .3526247171131696,
                              .5471536263305554, .7342101772154105, .8853209468390958, .9775206135612875};
        const double xx[8] = {.5, .1666666666666667, .08333333333333333, .05, .03333333333333333,
                              .02380952380952381, .01785714285714286, .01388888888888889};
        const double vv[7] = {.5, .3333333333333333, .25, .2, .1666666666666667, .1428571428571429, .125};
        for (int k = 0; k < 8; ++k) { h[k] = hh[k]; xc[k] = xx[k]; }
        for (int k = 0; k < 7; ++k) vc[k] = vv[k];
        int n = 0;
        for (int j = 1; j < 8; ++j)
            for (int k = 0; k < j; ++k) r[n++] = 1.0 / (h[j] - h[k]);
        // c/d in Fortran 1-based indexing n = 1..21 (stored at n-1)
        double C[22], D[22];
        C[1] = -h[1];
        D[1] = h[1];
        n = 1;
        for (int j = 3; j <= 7; ++j) {
            ++n;
            C[n] = -h[j - 1] * C[n - j + 2];
            D[n] = h[1] * D[n - j + 2];
            for (int k = 3; k <= j - 1; ++k) {
                ++n;
                C[n] = C[n - j + 1] - h[j - 1] * C[n - j + 2];
                D[n] = D[n - j + 1] + h[k - 1] * D[n - j + 2];
            }
            ++n;
            C[n] = C[n - j + 1] - h[j - 1];
            D[n] = D[n - j + 1] + h[j - 1];
        }
        for (int k = 0; k < 21; ++k) { c[k] = C[k + 1]; d[k] = D[k + 1]; }
    }
};

// Saved state of mdt_ra15 between calls: b, e (7 per coordinate) and dtflag.
struct Ra15State {
    std::vector<double> b, e;  // [3*nbod][7]
    int dtflag = 0;
    void size(int nbod) {
        if ((int)b.size() < 21 * nbod) {
            b.assign(21 * (size_t)nbod, 0.0);
            e.assign(21 * (size_t)nbod, 0.0);
        }
    }
};

// mdt_ra15, mercury6_2.for:4133-4485, with force = mfo_all. t is the trial
// sequence length (in/out: the next one on return), tdid the length done.
// Returns nonzero on a force failure or a non-finite predictor.
inline int mdt_ra15(double time, double& t, double& tdid, double tol, const double* jcen, int nbod, int nbig,
                    const double* mass, double* x1, double* v1, const double* ngf, int ngflag, int pn,
                    Ra15State& st, long long* forces) {
    static const Ra15Constants K;
    const double *h = K.h, *xc = K.xc, *vc = K.vc, *r = K.r, *c = K.c, *d = K.d;
    st.size(nbod);
    if (st.dtflag == 0) st.dtflag = 1;
    const int nv = 3 * nbod;
    std::vector<double> x(nv), v(nv), a(nv), a1(nv), g(7 * (size_t)nv);
    double* b = st.b.data();
    double* e = st.e.data();
    // Fortran arrays g(7,3n), b(7,3n): index [k*7 + m] for coordinate k (0-based), m = 0..6
    auto B = [&](int m, int k) -> double& { return b[(size_t)k * 7 + m]; };
    auto E = [&](int m, int k) -> double& { return e[(size_t)k * 7 + m]; };
    auto G = [&](int m, int k) -> double& { return g[(size_t)k * 7 + m]; };
    const bool vpred = (ngflag != 0 || pn == 1);
    for (;;) {
        int niter;
        if (st.dtflag == 1) {
            niter = 6;
            for (int k = 3; k < nv; ++k)
                for (int m = 0; m < 7; ++m) { B(m, k) = 0.0; E(m, k) = 0.0; }
        } else {
            niter = 2;
        }
        if (mfo_all(jcen, nbod, nbig, mass, x1, v1, a1.data(), ngf, ngflag, pn)) return 1;
        if (forces) ++*forces;
        for (int k = 3; k < nv; ++k) {
            G(0, k) = B(6, k) * d[15] + B(5, k) * d[10] + B(4, k) * d[6] + B(3, k) * d[3] + B(2, k) * d[1] +
                      B(1, k) * d[0] + B(0, k);
            G(1, k) = B(6, k) * d[16] + B(5, k) * d[11] + B(4, k) * d[7] + B(3, k) * d[4] + B(2, k) * d[2] + B(1, k);
            G(2, k) = B(6, k) * d[17] + B(5, k) * d[12] + B(4, k) * d[8] + B(3, k) * d[5] + B(2, k);
            G(3, k) = B(6, k) * d[18] + B(5, k) * d[13] + B(4, k) * d[9] + B(3, k);
            G(4, k) = B(6, k) * d[19] + B(5, k) * d[14] + B(4, k);
            G(5, k) = B(6, k) * d[20] + B(5, k);
            G(6, k) = B(6, k);
        }
        double s[9];
        for (int n = 1; n <= niter; ++n) {
            for (int j = 2; j <= 8; ++j) {
                const double hj = h[j - 1];
                s[0] = t * hj;
                s[1] = s[0] * s[0] * .5;
                s[2] = s[1] * hj * .3333333333333333;
                s[3] = s[2] * hj * .5;
                s[4] = s[3] * hj * .6;
                s[5] = s[4] * hj * .6666666666666667;
                s[6] = s[5] * hj * .7142857142857143;
                s[7] = s[6] * hj * .75;
                s[8] = s[7] * hj * .7777777777777778;
                for (int k = 3; k < nv; ++k)
                    x[k] = s[8] * B(6, k) + s[7] * B(5, k) + s[6] * B(4, k) + s[5] * B(3, k) + s[4] * B(2, k) +
                           s[3] * B(1, k) + s[2] * B(0, k) + s[1] * a1[k] + s[0] * v1[k] + x1[k];
                if (vpred) {
                    s[0] = t * hj;
                    s[1] = s[0] * hj * .5;
                    s[2] = s[1] * hj * .6666666666666667;
                    s[3] = s[2] * hj * .75;
                    s[4] = s[3] * hj * .8;
                    s[5] = s[4] * hj * .8333333333333333;
                    s[6] = s[5] * hj * .8571428571428571;
                    s[7] = s[6] * hj * .875;
                    for (int k = 3; k < nv; ++k)
                        v[k] = s[7] * B(6, k) + s[6] * B(5, k) + s[5] * B(4, k) + s[4] * B(3, k) + s[3] * B(2, k) +
                               s[2] * B(1, k) + s[1] * B(0, k) + s[0] * a1[k] + v1[k];
                }
                // the central body's entries (k < 3) of the predictors stay as copied
                for (int k = 0; k < 3; ++k) { x[k] = x1[k]; v[k] = v1[k]; }
                if (mfo_all(jcen, nbod, nbig, mass, x.data(), vpred ? v.data() : v1, a.data(), ngf, ngflag, pn))
                    return 1;
                if (forces) ++*forces;
                for (int k = 3; k < nv; ++k) {
                    const double gk = a[k] - a1[k];
                    double temp;
                    switch (j) {
                    case 2:
                        temp = G(0, k);
                        G(0, k) = (a[k] - a1[k]) * r[0];
                        B(0, k) = B(0, k) + G(0, k) - temp;
                        break;
                    case 3:
                        temp = G(1, k);
                        G(1, k) = (gk * r[1] - G(0, k)) * r[2];
                        temp = G(1, k) - temp;
                        B(0, k) = B(0, k) + temp * c[0];
                        B(1, k) = B(1, k) + temp;
                        break;
                    case 4:
                        temp = G(2, k);
                        G(2, k) = ((gk * r[3] - G(0, k)) * r[4] - G(1, k)) * r[5];
                        temp = G(2, k) - temp;
                        B(0, k) = B(0, k) + temp * c[1];
                        B(1, k) = B(1, k) + temp * c[2];
                        B(2, k) = B(2, k) + temp;
                        break;
                    case 5:
                        temp = G(3, k);
                        G(3, k) = (((gk * r[6] - G(0, k)) * r[7] - G(1, k)) * r[8] - G(2, k)) * r[9];
                        temp = G(3, k) - temp;
                        B(0, k) = B(0, k) + temp * c[3];
                        B(1, k) = B(1, k) + temp * c[4];
                        B(2, k) = B(2, k) + temp * c[5];
                        B(3, k) = B(3, k) + temp;
                        break;
                    case 6:
                        temp = G(4, k);
                        G(4, k) = ((((gk * r[10] - G(0, k)) * r[11] - G(1, k)) * r[12] - G(2, k)) * r[13] - G(3, k)) *
                                  r[14];
                        temp = G(4, k) - temp;
                        B(0, k) = B(0, k) + temp * c[6];
                        B(1, k) = B(1, k) + temp * c[7];
                        B(2, k) = B(2, k) + temp * c[8];
                        B(3, k) = B(3, k) + temp * c[9];
                        B(4, k) = B(4, k) + temp;
                        break;
                    case 7:
                        temp = G(5, k);
                        G(5, k) = (((((gk * r[15] - G(0, k)) * r[16] - G(1, k)) * r[17] - G(2, k)) * r[18] - G(3, k)) *
                                       r[19] -
                                   G(4, k)) *
                                  r[20];
                        temp = G(5, k) - temp;
                        B(0, k) = B(0, k) + temp * c[10];
                        B(1, k) = B(1, k) + temp * c[11];
                        B(2, k) = B(2, k) + temp * c[12];
                        B(3, k) = B(3, k) + temp * c[13];
                        B(4, k) = B(4, k) + temp * c[14];
                        B(5, k) = B(5, k) + temp;
                        break;
                    default:
                        temp = G(6, k);
                        G(6, k) = ((((((gk * r[21] - G(0, k)) * r[22] - G(1, k)) * r[23] - G(2, k)) * r[24] - G(3, k)) *
                                        r[25] -
                                    G(4, k)) *
                                       r[26] -
                                   G(5, k)) *
                                  r[27];
                        temp = G(6, k) - temp;
                        B(0, k) = B(0, k) + temp * c[15];
                        B(1, k) = B(1, k) + temp * c[16];
                        B(2, k) = B(2, k) + temp * c[17];
                        B(3, k) = B(3, k) + temp * c[18];
                        B(4, k) = B(4, k) + temp * c[19];
                        B(5, k) = B(5, k) + temp * c[20];
                        B(6, k) = B(6, k) + temp;
                        break;
                    }
                }
            }
        }
        double temp = 0.0;
        for (int k = 3; k < nv; ++k) {
            if (!std::isfinite(B(6, k))) return 1;
            temp = std::max(temp, std::fabs(B(6, k)));
        }
        temp = temp / (72.0 * std::pow(std::fabs(t), 7.0));
        tdid = t;
        if (temp == 0.0) t = tdid * 1.4;
        else t = std::copysign(std::pow(tol / temp, 1.0 / 9.0), tdid);
        if (st.dtflag == 1 && std::fabs(t / tdid) < 1.0) {
            t = t * .8;
            continue;
        }
        if (std::fabs(t / tdid) > 1.4) t = tdid * 1.4;
        temp = tdid * tdid;
        for (int k = 3; k < nv; ++k) {
            x1[k] = (xc[7] * B(6, k) + xc[6] * B(5, k) + xc[5] * B(4, k) + xc[4] * B(3, k) + xc[3] * B(2, k) +
                     xc[2] * B(1, k) + xc[1] * B(0, k) + xc[0] * a1[k]) *
                        temp +
                    v1[k] * tdid + x1[k];
            v1[k] = (vc[6] * B(6, k) + vc[5] * B(5, k) + vc[4] * B(4, k) + vc[3] * B(3, k) + vc[2] * B(2, k) +
                     vc[1] * B(1, k) + vc[0] * B(0, k) + a1[k]) *
                        tdid +
                    v1[k];
        }
        const double q = t / tdid;
        const double q2 = q * q, q3 = q * q2, q4 = q2 * q2, q5 = q2 * q3, q6 = q3 * q3, q7 = q3 * q4;
        for (int k = 3; k < nv; ++k) {
            double sv[7];
            for (int m = 0; m < 7; ++m) sv[m] = B(m, k) - E(m, k);
            if (st.dtflag == 1)
                for (int m = 0; m < 7; ++m) sv[m] = 0.0;
            E(0, k) = q * (B(6, k) * 7.0 + B(5, k) * 6.0 + B(4, k) * 5.0 + B(3, k) * 4.0 + B(2, k) * 3.0 +
                           B(1, k) * 2.0 + B(0, k));
            E(1, k) = q2 * (B(6, k) * 21.0 + B(5, k) * 15.0 + B(4, k) * 10.0 + B(3, k) * 6.0 + B(2, k) * 3.0 + B(1, k));
            E(2, k) = q3 * (B(6, k) * 35.0 + B(5, k) * 20.0 + B(4, k) * 10.0 + B(3, k) * 4.0 + B(2, k));
            E(3, k) = q4 * (B(6, k) * 35.0 + B(5, k) * 15.0 + B(4, k) * 5.0 + B(3, k));
            E(4, k) = q5 * (B(6, k) * 21.0 + B(5, k) * 6.0 + B(4, k));
            E(5, k) = q6 * (B(6, k) * 7.0 + B(5, k));
            E(6, k) = q7 * B(6, k);
            for (int m = 0; m < 7; ++m) B(m, k) = E(m, k) + sv[m];
        }
        st.dtflag = 2;
        return 0;
    }
}

}  // namespace oracle
