// Test infrastructure only: CPU restatement of MERCURY6's Bulirsch-Stoer
// integrators mdt_bs1 (modified midpoint, 8 levels) and mdt_bs2 (conservative
// Stoermer form, 12 levels), statement for statement, with force = mfo_all.
#pragma once
#include <algorithm>
#include <cmath>
#include <vector>

#include "oracle_ra15.hpp"

namespace oracle {

constexpr double BS_SHRINK = 0.55, BS_GROW = 1.3;

// The error test shared by both routines (mercury6_2.for:3369-3380,
// 3557-3568): max over bodies of the squared last extrapolation term scaled by
// 1/R^2 and 1/V^2. Returns false when a term is not finite (the Fortran fails).
template <class R>
bool bs_error(int nbod, const std::vector<R>& d1, const std::vector<double>& xscal, const std::vector<double>& vscal,
              double& errmax) {
    errmax = 0.0;
    for (int k = 1; k < nbod; ++k) {
        double q[6];
        for (int c = 0; c < 6; ++c) q[c] = val(d1[6 * (size_t)k + c]);
        for (int c = 0; c < 6; ++c)
            if (!std::isfinite(q[c])) return false;
        const double tmp1 = std::max(std::max(q[0] * q[0], q[1] * q[1]), q[2] * q[2]);
        const double tmp2 = std::max(std::max(q[3] * q[3], q[4] * q[4]), q[5] * q[5]);
        errmax = std::max(std::max(errmax, tmp1 * xscal[k]), tmp2 * vscal[k]);
    }
    return true;
}

// Neville update of the extrapolation table after level n (1-based), the
// loop both routines share (mercury6_2.for:3352-3366, 3540-3554).
template <class R> void bs_extrapolate(int nbod, int n, const double* h2, std::vector<std::vector<R>>& d) {
    for (int j = n - 1; j >= 1; --j) {
        const int j1 = j + 1;
        const double tmp0 = 1.0 / (h2[j] - h2[n]);
        const double tmp1 = tmp0 * h2[j1];
        const double tmp2 = tmp0 * h2[n];
        for (int k = 1; k < nbod; ++k)
            for (int c = 0; c < 6; ++c)
                d[j][6 * k + c] = R(tmp1) * d[j1][6 * k + c] - R(tmp2) * d[j][6 * k + c];
    }
}

template <class R> void bs_accept(int nbod, int n, const std::vector<std::vector<R>>& d, R* x0, R* v0) {
    for (int k = 1; k < nbod; ++k)
        for (int c = 0; c < 3; ++c) {
            x0[3 * k + c] = d[1][6 * k + c];
            v0[3 * k + c] = d[1][6 * k + 3 + c];
        }
    for (int j = 2; j <= n; ++j)
        for (int k = 1; k < nbod; ++k)
            for (int c = 0; c < 3; ++c) {
                x0[3 * k + c] = x0[3 * k + c] + d[j][6 * k + c];
                v0[3 * k + c] = v0[3 * k + c] + d[j][6 * k + 3 + c];
            }
}

template <class R>
void bs_scales(int nbod, const R* x0, const R* v0, std::vector<double>& xscal, std::vector<double>& vscal) {
    for (int k = 1; k < nbod; ++k) {
        const double p[3] = {val(x0[3 * k]), val(x0[3 * k + 1]), val(x0[3 * k + 2])};
        const double u[3] = {val(v0[3 * k]), val(v0[3 * k + 1]), val(v0[3 * k + 2])};
        const double tmp1 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
        const double tmp2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        xscal[k] = 1.0 / std::max(tmp1, 1e-300);
        vscal[k] = 1.0 / std::max(tmp2, 1e-300);
    }
}

// mdt_bs1, mercury6_2.for:3227-3404. h0 in/out (the next step on return),
// hdid the step done; *rejected counts halvings. Returns nonzero on a fail().
inline int mdt_bs1(double time, double& h0, double& hdid, double tol, const double* jcen, int nbod, int nbig,
                   const double* mass, double* x0, double* v0, const double* ngf, int ngflag, int pn,
                   long long* forces, long long* rejected) {
    (void)time;
    const double tol2 = tol * tol;
    const size_t nv = 3 * (size_t)nbod;
    std::vector<double> xscal(nbod), vscal(nbod), x(nv), v(nv), xend(nv), vend(nv), a(nv), a0(nv);
    std::vector<std::vector<double>> d(9, std::vector<double>(6 * (size_t)nbod));
    double h2[9];
    bs_scales(nbod, x0, v0, xscal, vscal);
    auto force = [&](const double* xx, const double* vv, double* aa) {
        if (forces) ++*forces;
        return mfo_all(jcen, nbod, nbig, mass, xx, vv, aa, ngf, ngflag, pn);
    };
    if (force(x0, v0, a0.data())) return 1;
    for (;;) {
        if (time + h0 == time) return 1;
        for (int n = 1; n <= 8; ++n) {
            const double h = h0 / (2.0 * double(n));
            h2[n] = 0.25 / double(n * n);
            const double hx2 = h * 2.0;
            for (size_t k = 3; k < nv; ++k) {
                x[k] = x0[k] + h * v0[k];
                v[k] = v0[k] + h * a0[k];
            }
            if (force(x.data(), v.data(), a.data())) return 1;
            for (size_t k = 3; k < nv; ++k) {
                xend[k] = x0[k] + hx2 * v[k];
                vend[k] = v0[k] + hx2 * a[k];
            }
            for (int j = 2; j <= n; ++j) {
                if (force(xend.data(), vend.data(), a.data())) return 1;
                for (size_t k = 3; k < nv; ++k) {
                    x[k] = x[k] + hx2 * vend[k];
                    v[k] = v[k] + hx2 * a[k];
                }
                if (force(x.data(), v.data(), a.data())) return 1;
                for (size_t k = 3; k < nv; ++k) {
                    xend[k] = xend[k] + hx2 * v[k];
                    vend[k] = vend[k] + hx2 * a[k];
                }
            }
            if (force(xend.data(), vend.data(), a.data())) return 1;
            for (int k = 1; k < nbod; ++k)
                for (int c = 0; c < 3; ++c) {
                    const size_t z = 3 * (size_t)k + c;
                    d[n][6 * k + c] = 0.5 * (xend[z] + x[z] + h * vend[z]);
                    d[n][6 * k + 3 + c] = 0.5 * (vend[z] + v[z] + h * a[z]);
                }
            bs_extrapolate(nbod, n, h2, d);
            if (n > 3) {
                double errmax;
                if (!bs_error(nbod, d[1], xscal, vscal, errmax)) return 1;
                if (errmax <= tol2) {
                    bs_accept(nbod, n, d, x0, v0);
                    hdid = h0;
                    if (n == 8) h0 = h0 * BS_SHRINK;
                    if (n < 7) h0 = h0 * BS_GROW;
                    return 0;
                }
            }
        }
        if (rejected) ++*rejected;
        h0 = h0 * 0.5;
    }
}

// mdt_bs2, mercury6_2.for:3428-3596, with any force routine
// force(x, v, a) -> nonzero on fail(); the force is evaluated with the
// start-of-step velocities v0 (conservative systems). The state may be any
// scalar type R (dual numbers propagate tangents); the step control reads the
// values only.
template <class R, class Force>
int mdt_bs2_with(Force&& force, double time, double& h0, double& hdid, double tol, int nbod, R* x0, R* v0,
                 long long* rejected) {
    const double tol2 = tol * tol;
    const size_t nv = 3 * (size_t)nbod;
    std::vector<double> xscal(nbod), vscal(nbod);
    std::vector<R> xend(nv), a(nv), a0(nv), b(nv), c(nv);
    std::vector<std::vector<R>> d(13, std::vector<R>(6 * (size_t)nbod));
    double h2[13];
    bs_scales(nbod, x0, v0, xscal, vscal);
    if (force(x0, v0, a0.data())) return 1;
    for (;;) {
        if (time + h0 == time) return 1;
        for (int n = 1; n <= 12; ++n) {
            const double h = h0 / double(n);
            const double hby2 = 0.5 * h;
            h2[n] = h * h;
            const double h2by2 = 0.5 * h2[n];
            for (size_t k = 3; k < nv; ++k) {
                b[k] = R(0.5) * a0[k];
                c[k] = R(0.0);
                xend[k] = R(h2by2) * a0[k] + R(h) * v0[k] + x0[k];
            }
            for (int j = 2; j <= n; ++j) {
                if (force(xend.data(), v0, a.data())) return 1;
                const double tmp0 = h * double(j);
                for (size_t k = 3; k < nv; ++k) {
                    b[k] = b[k] + a[k];
                    c[k] = c[k] + b[k];
                    xend[k] = R(h2[n]) * c[k] + R(h2by2) * a0[k] + R(tmp0) * v0[k] + x0[k];
                }
            }
            if (force(xend.data(), v0, a.data())) return 1;
            for (int k = 1; k < nbod; ++k)
                for (int q = 0; q < 3; ++q) {
                    const size_t z = 3 * (size_t)k + q;
                    d[n][6 * k + q] = xend[z];
                    d[n][6 * k + 3 + q] = R(h) * b[z] + R(hby2) * a[z] + v0[z];
                }
            bs_extrapolate(nbod, n, h2, d);
            if (n > 3) {
                double errmax;
                if (!bs_error(nbod, d[1], xscal, vscal, errmax)) return 1;
                if (errmax <= tol2) {
                    bs_accept(nbod, n, d, x0, v0);
                    hdid = h0;
                    if (n >= 8) h0 = h0 * BS_SHRINK;
                    if (n < 7) h0 = h0 * BS_GROW;
                    return 0;
                }
            }
        }
        if (rejected) ++*rejected;
        h0 = h0 * 0.5;
    }
}

inline int mdt_bs2(double time, double& h0, double& hdid, double tol, const double* jcen, int nbod, int nbig,
                   const double* mass, double* x0, double* v0, const double* ngf, int ngflag, int pn,
                   long long* forces, long long* rejected) {
    auto force = [&](const double* xx, const double* vv, double* aa) {
        if (forces) ++*forces;
        return mfo_all(jcen, nbod, nbig, mass, xx, vv, aa, ngf, ngflag, pn);
    };
    return mdt_bs2_with(force, time, h0, hdid, tol, nbod, x0, v0, rejected);
}

}  // namespace oracle
