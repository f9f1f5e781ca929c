// Test infrastructure only: the energy and angular-momentum check of
// MERCURY6, restated statement for statement from the Fortran.
//   mco_h2b  mercury6_2.for:2348-2405  heliocentric -> barycentric
//   mxx_en   mercury6_2.for:7226-7315  energy e and |L| of all nbod bodies
// Arrays use the Fortran layout: x(3,nbod) as rows of three.
#pragma once
#include <cmath>
#include <vector>

namespace oracle {

// mco_h2b: x, v (3, n) barycentric from xh, vh.
template <class R>
void mco_h2b(int n, const R* m, const R* xh, const R* vh, R* x, R* v) {
    R mtot(0.0);
    for (int c = 0; c < 3; ++c) {
        x[c] = R(0.0);
        v[c] = R(0.0);
    }
    for (int j = 1; j < n; ++j) {
        mtot = mtot + m[j];
        for (int c = 0; c < 3; ++c) {
            x[c] = x[c] + m[j] * xh[3 * j + c];
            v[c] = v[c] + m[j] * vh[3 * j + c];
        }
    }
    const R temp = R(-1.0) / (mtot + m[0]);
    for (int c = 0; c < 3; ++c) {
        x[c] = temp * x[c];
        v[c] = temp * v[c];
    }
    for (int j = 1; j < n; ++j)
        for (int c = 0; c < 3; ++c) {
            x[3 * j + c] = xh[3 * j + c] + x[c];
            v[3 * j + c] = vh[3 * j + c] + v[c];
        }
}

// mxx_en: energy e and angular momentum magnitude l2 (spin s may be null).
template <class R>
void mxx_en(const R* jcen, int n, const R* m, const R* xh, const R* vh, const R* s, R& e, R& l2) {
    std::vector<R> x(3 * (size_t)n), v(3 * (size_t)n);
    R ke(0.0), pe(0.0), l[3] = {R(0.0), R(0.0), R(0.0)};
    mco_h2b(n, m, xh, vh, x.data(), v.data());
    if (s)
        for (int j = 0; j < n; ++j)
            for (int c = 0; c < 3; ++c) l[c] = l[c] + s[3 * j + c];
    for (int j = 0; j < n; ++j) {
        const R* xj = &x[3 * (size_t)j];
        const R* vj = &v[3 * (size_t)j];
        l[0] = l[0] + m[j] * (xj[1] * vj[2] - xj[2] * vj[1]);
        l[1] = l[1] + m[j] * (xj[2] * vj[0] - xj[0] * vj[2]);
        l[2] = l[2] + m[j] * (xj[0] * vj[1] - xj[1] * vj[0]);
        ke = ke + m[j] * (vj[0] * vj[0] + vj[1] * vj[1] + vj[2] * vj[2]);
    }
    for (int j = 1; j < n; ++j) {
        if (m[j] == R(0.0)) continue;
        R tmp(0.0);
        for (int k = j + 1; k < n; ++k) {
            if (m[k] == R(0.0)) continue;
            const R dx = x[3 * k] - x[3 * j];
            const R dy = x[3 * k + 1] - x[3 * j + 1];
            const R dz = x[3 * k + 2] - x[3 * j + 2];
            const R r2 = dx * dx + dy * dy + dz * dz;
            if (r2 != R(0.0)) tmp = tmp + m[k] / std::sqrt(r2);
        }
        pe = pe - tmp * m[j];
    }
    for (int j = 1; j < n; ++j) {
        const R dx = x[3 * j] - x[0];
        const R dy = x[3 * j + 1] - x[1];
        const R dz = x[3 * j + 2] - x[2];
        const R r2 = dx * dx + dy * dy + dz * dz;
        if (r2 != R(0.0)) pe = pe - m[0] * m[j] / std::sqrt(r2);
    }
    if (jcen[0] != R(0.0) || jcen[1] != R(0.0) || jcen[2] != R(0.0)) {
        for (int j = 1; j < n; ++j) {
            const R* p = &xh[3 * (size_t)j];
            const R r2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
            const R r_1 = R(1.0) / std::sqrt(r2);
            const R r_2 = r_1 * r_1;
            const R r_4 = r_2 * r_2;
            const R r_6 = r_4 * r_2;
            const R u2 = p[2] * p[2] * r_2;
            const R u4 = u2 * u2;
            const R u6 = u4 * u2;
            pe = pe + m[0] * m[j] * r_1 *
                          (jcen[0] * r_2 * (R(1.5) * u2 - R(0.5)) +
                           jcen[1] * r_4 * (R(4.375) * u4 - R(3.75) * u2 + R(0.375)) +
                           jcen[2] * r_6 * (R(14.4375) * u6 - R(19.6875) * u4 + R(6.5625) * u2 - R(0.3125)));
        }
    }
    e = R(0.5) * ke + pe;
    l2 = std::sqrt(l[0] * l[0] + l[1] * l[1] + l[2] * l[2]);
}

}  // namespace oracle
