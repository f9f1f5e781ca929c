// Test infrastructure only: CPU restatement of MERCURY6's hybrid symplectic
// step (mdt_hy) with its changeover forces (mfo_drct, mfo_hy, mfo_hkce), the
// encounter sniffer (mce_snif), the democratic-heliocentric conversions
// (mco_dh2h, mco_h2dh) and the close-encounter subsystem (mdt_hkce, BS2 with
// mfo_hkce and mce_stat per substep), statement for statement.
//
// mdt_hkce's collision branch (mce_coll, only with collisions enabled) is not
// restated: the reference's CUDA path hands collisions to the Fortran host
// too, and the hit records themselves are produced.
#pragma once
#include <algorithm>
#include <cmath>
#include <vector>

#include "oracle_bs.hpp"
#include "oracle_mvs.hpp"

namespace oracle {

// mfo_drct, mercury6_2.for:4708-4765: direct terms between Big i >= i0 and
// every j > i with the changeover K(r) = 10q^3 - 15q^4 + 6q^5 (0 inside
// 0.1 rc, 1 outside rc).
template <class R>
void mfo_drct(int i0, int nbod, int nbig, const R* m, const R* x, const double* rcrit, R* a) {
    if (i0 <= 0) i0 = 1;
    for (int i = i0; i < nbig; ++i)
        for (int j = i + 1; j < nbod; ++j) {
            const R dx = x[3 * j] - x[3 * i];
            const R dy = x[3 * j + 1] - x[3 * i + 1];
            const R dz = x[3 * j + 2] - x[3 * i + 2];
            const R s2 = dx * dx + dy * dy + dz * dz;
            const double rc = std::max(rcrit[i], rcrit[j]);
            const double rc2 = rc * rc;
            R tmp2;
            if (s2 >= R(rc2)) {
                const R s_1 = R(1.0) / Sqrt(s2);
                tmp2 = s_1 * s_1 * s_1;
            } else if (s2 <= R(0.01 * rc2)) {
                tmp2 = R(0.0);
            } else {
                const R s_1 = R(1.0) / Sqrt(s2);
                const R s = R(1.0) / s_1;
                const R s_3 = s_1 * s_1 * s_1;
                const R q = (s - R(0.1 * rc)) / R(0.9 * rc);
                const R q2 = q * q, q3 = q * q2, q4 = q2 * q2, q5 = q2 * q3;
                tmp2 = (R(10.0) * q3 - R(15.0) * q4 + R(6.0) * q5) * s_3;
            }
            const R faci = tmp2 * m[i];
            const R facj = tmp2 * m[j];
            a[3 * j] = a[3 * j] - faci * dx;
            a[3 * j + 1] = a[3 * j + 1] - faci * dy;
            a[3 * j + 2] = a[3 * j + 2] - faci * dz;
            a[3 * i] = a[3 * i] + facj * dx;
            a[3 * i + 1] = a[3 * i + 1] + facj * dy;
            a[3 * i + 2] = a[3 * i + 2] + facj * dz;
        }
}

// mfo_hy, mercury6_2.for:4781-4819: the interaction part of the hybrid
// Hamiltonian (no indirect term in democratic heliocentric coordinates).
template <class R>
void mfo_hy(const double* jcen, int nbod, int nbig, const R* m, const R* x, const double* rcrit, R* a) {
    for (int k = 0; k < 3 * nbod; ++k) a[k] = R(0.0);
    mfo_drct(1, nbod, nbig, m, x, rcrit, a);
    if (jcen[0] != 0.0 || jcen[1] != 0.0 || jcen[2] != 0.0) {
        std::vector<R> aobl(3 * (size_t)nbod);
        R acen[3];
        mfo_obl(jcen, nbod, m, x, aobl.data(), acen);
        for (int k = 1; k < nbod; ++k)
            for (int c = 0; c < 3; ++c) a[3 * k + c] = a[3 * k + c] + aobl[3 * k + c] - acen[c];
    }
}

// mfo_hkce, mercury6_2.for:4836-4910: the Keplerian part during encounters:
// the inner changeover 1 - K(r) over the listed pairs (0-based ice, jce)
// plus the central body's attraction.
template <class R>
void mfo_hkce(int nbod, const R* m, const R* x, const double* rcrit, R* a, int nce, const int* ice, const int* jce) {
    for (int k = 0; k < 3 * nbod; ++k) a[k] = R(0.0);
    for (int k = 0; k < nce; ++k) {
        const int i = ice[k], j = jce[k];
        const R dx = x[3 * j] - x[3 * i];
        const R dy = x[3 * j + 1] - x[3 * i + 1];
        const R dz = x[3 * j + 2] - x[3 * i + 2];
        const R s2 = dx * dx + dy * dy + dz * dz;
        const double rc = std::max(rcrit[i], rcrit[j]);
        const double rc2 = rc * rc;
        if (s2 < R(rc2)) {
            const R s_1 = R(1.0) / Sqrt(s2);
            const R s_3 = s_1 * s_1 * s_1;
            R tmp2;
            if (s2 <= R(0.01 * rc2)) {
                tmp2 = s_3;
            } else {
                const R s = R(1.0) / s_1;
                const R q = (s - R(0.1 * rc)) / R(0.9 * rc);
                const R q2 = q * q, q3 = q * q2, q4 = q2 * q2, q5 = q2 * q3;
                tmp2 = (R(1.0) - R(10.0) * q3 + R(15.0) * q4 - R(6.0) * q5) * s_3;
            }
            const R faci = tmp2 * m[i];
            const R facj = tmp2 * m[j];
            a[3 * j] = a[3 * j] - faci * dx;
            a[3 * j + 1] = a[3 * j + 1] - faci * dy;
            a[3 * j + 2] = a[3 * j + 2] - faci * dz;
            a[3 * i] = a[3 * i] + facj * dx;
            a[3 * i + 1] = a[3 * i + 1] + facj * dy;
            a[3 * i + 2] = a[3 * i + 2] + facj * dz;
        }
    }
    for (int i = 1; i < nbod; ++i) {
        const R s2 = x[3 * i] * x[3 * i] + x[3 * i + 1] * x[3 * i + 1] + x[3 * i + 2] * x[3 * i + 2];
        const R s_1 = R(1.0) / Sqrt(s2);
        const R tmp2 = m[0] * s_1 * s_1 * s_1;
        a[3 * i] = a[3 * i] - tmp2 * x[3 * i];
        a[3 * i + 1] = a[3 * i + 1] - tmp2 * x[3 * i + 1];
        a[3 * i + 2] = a[3 * i + 2] - tmp2 * x[3 * i + 2];
    }
}

// mce_snif, mercury6_2.for:1648-1734 (i0 = 2): pairs (Big i, j > i) whose
// separation came within max(rcrit) during the drift; 0-based ice/jce in
// i-outer j-inner order, ce[j] = 2 for every member.
inline void mce_snif(double h, int nbod, int nbig, const double* x0, const double* v0, const double* x1,
                     const double* v1, const double* rcrit, std::vector<int>& ce, std::vector<int>& ice,
                     std::vector<int>& jce) {
    ce.assign(nbod, 0);
    ice.clear();
    jce.clear();
    std::vector<double> xmin(nbod), xmax(nbod), ymin(nbod), ymax(nbod);
    mce_box(nbod, h, x0, v0, x1, v1, xmin.data(), xmax.data(), ymin.data(), ymax.data());
    for (int j = 1; j < nbig; ++j) {
        xmin[j] = xmin[j] - rcrit[j];
        xmax[j] = xmax[j] + rcrit[j];
        ymin[j] = ymin[j] - rcrit[j];
        ymax[j] = ymax[j] + rcrit[j];
    }
    for (int i = 1; i < nbig; ++i)
        for (int j = i + 1; j < nbod; ++j) {
            if (!(xmax[i] >= xmin[j] && xmax[j] >= xmin[i] && ymax[i] >= ymin[j] && ymax[j] >= ymin[i])) continue;
            const double rc = std::max(rcrit[i], rcrit[j]);
            const double rc2 = rc * rc;
            const double dx0 = x0[3 * i] - x0[3 * j], dy0 = x0[3 * i + 1] - x0[3 * j + 1],
                         dz0 = x0[3 * i + 2] - x0[3 * j + 2];
            const double dx1 = x1[3 * i] - x1[3 * j], dy1 = x1[3 * i + 1] - x1[3 * j + 1],
                         dz1 = x1[3 * i + 2] - x1[3 * j + 2];
            const double d0 = dx0 * dx0 + dy0 * dy0 + dz0 * dz0;
            const double d1 = dx1 * dx1 + dy1 * dy1 + dz1 * dz1;
            const double du0 = v0[3 * i] - v0[3 * j], dv0 = v0[3 * i + 1] - v0[3 * j + 1],
                         dw0 = v0[3 * i + 2] - v0[3 * j + 2];
            const double du1 = v1[3 * i] - v1[3 * j], dv1 = v1[3 * i + 1] - v1[3 * j + 1],
                         dw1 = v1[3 * i + 2] - v1[3 * j + 2];
            const double d0t = (dx0 * du0 + dy0 * dv0 + dz0 * dw0) * 2.0;
            const double d1t = (dx1 * du1 + dy1 * dv1 + dz1 * dw1) * 2.0;
            double d2min = HUGE_, tmin;
            if (d0t * h <= 0.0 && d1t * h >= 0.0) mce_min(d0, d1, d0t, d1t, h, d2min, tmin);
            const double temp = std::min(std::min(d0, d1), d2min);
            if (temp <= rc2) {
                ce[i] = 2;
                ce[j] = 2;
                ice.push_back(i);
                jce.push_back(j);
            }
        }
}

// mco_dh2h velocities, mercury6_2.for:2007-2051 (positions are unchanged).
inline void dh2h_velocity(int nbod, const double* m, const double* v, double* vh) {
    double mvsum[3] = {0.0, 0.0, 0.0};
    for (int j = 1; j < nbod; ++j)
        for (int c = 0; c < 3; ++c) mvsum[c] = mvsum[c] + m[j] * v[3 * j + c];
    const double temp = 1.0 / m[0];
    for (int c = 0; c < 3; ++c) mvsum[c] = temp * mvsum[c];
    for (int c = 0; c < 3; ++c) vh[c] = v[c];
    for (int j = 1; j < nbod; ++j)
        for (int c = 0; c < 3; ++c) vh[3 * j + c] = v[3 * j + c] + mvsum[c];
}

// mco_h2dh, mercury6_2.for:2550-2596.
inline void h2dh_velocity(int nbod, const double* m, const double* vh, double* v) {
    double mtot = 0.0, mvsum[3] = {0.0, 0.0, 0.0};
    for (int j = 1; j < nbod; ++j) {
        mtot = mtot + m[j];
        for (int c = 0; c < 3; ++c) mvsum[c] = mvsum[c] + m[j] * vh[3 * j + c];
    }
    const double temp = 1.0 / (m[0] + mtot);
    for (int c = 0; c < 3; ++c) mvsum[c] = temp * mvsum[c];
    for (int c = 0; c < 3; ++c) v[c] = vh[c];
    for (int j = 1; j < nbod; ++j)
        for (int c = 0; c < 3; ++c) v[3 * j + c] = vh[3 * j + c] - mvsum[c];
}

// The solar-drift half step of mdt_hy (mercury6_2.for:3693-3711).
template <class R> void solar_drift(int nbod, const R* m, R* x, const R* v, double hby2) {
    R mvsum[3] = {R(0.0), R(0.0), R(0.0)};
    for (int j = 1; j < nbod; ++j)
        for (int c = 0; c < 3; ++c) mvsum[c] = mvsum[c] + m[j] * v[3 * j + c];
    const R temp = R(hby2) / m[0];
    for (int c = 0; c < 3; ++c) mvsum[c] = temp * mvsum[c];
    for (int j = 1; j < nbod; ++j)
        for (int c = 0; c < 3; ++c) x[3 * j + c] = x[3 * j + c] + mvsum[c];
}

// State mdt_hy keeps between calls: the cached interaction and
// non-gravitational accelerations and the encounter step hrec.
template <class R> struct HyState {
    std::vector<R> a, angf;
    double hrec = 0.0;
    int dtflag = 0;
};

// mdt_hkce, mercury6_2.for:3798-3965 without the collision branch: the
// encounter members (ce != 0) and the central body integrated together by
// mdt_bs2 with mfo_hkce on a local clock, mce_stat after every substep.
// Event ids are mapped back to the global (1-based) numbering. Returns
// nonzero on a fail(). Any scalar type R: mce_stat reads the values.
template <class R>
int mdt_hkce(double time, double h0, double& hrec, double tol, int nbod, int nbig, const R* m, R* x, R* v,
             const double* rphys, const double* rcrit, const double* rce, const std::vector<int>& ce,
             const std::vector<int>& ice, const std::vector<int>& jce, std::vector<Event>& events, long long* forces) {
    std::vector<int> index(1, 0), iback(nbod, -1);
    int nbsbig = 0;
    for (int j = 1; j < nbod; ++j)
        if (ce[j] != 0) {
            if (j < nbig) nbsbig = (int)index.size();
            iback[j] = (int)index.size();
            index.push_back(j);
        }
    const int nbs = (int)index.size();
    nbsbig = nbsbig + 1;  // count of Big bodies incl. the central body
    std::vector<R> mbs(nbs), xbs(3 * (size_t)nbs, R(0.0)), vbs(3 * (size_t)nbs, R(0.0));
    std::vector<double> rcritbs(nbs, 0.0), rcebs(nbs, 0.0), rphybs(nbs, 0.0);
    mbs[0] = m[0];
    for (int k = 1; k < nbs; ++k) {
        const int j = index[k];
        mbs[k] = m[j];
        for (int c = 0; c < 3; ++c) {
            xbs[3 * k + c] = x[3 * j + c];
            vbs[3 * k + c] = v[3 * j + c];
        }
        rcebs[k] = rce[j];
        rphybs[k] = rphys[j];
        rcritbs[k] = rcrit[j];
    }
    const int nce = (int)ice.size();
    std::vector<int> ibs(nce), jbs(nce);
    for (int k = 0; k < nce; ++k) {
        ibs[k] = iback[ice[k]];
        jbs[k] = iback[jce[k]];
    }
    auto force = [&](const R* xx, const R*, R* aa) {
        if (forces) ++*forces;
        mfo_hkce(nbs, mbs.data(), xx, rcritbs.data(), aa, nce, ibs.data(), jbs.data());
        return 0;
    };
    double tlocal = 0.0;
    double hlocal = std::copysign(hrec, h0);
    std::vector<R> x0(3 * (size_t)nbs), v0(3 * (size_t)nbs);
    std::vector<double> mv(nbs), x0v(3 * (size_t)nbs), v0v(3 * (size_t)nbs), x1v(3 * (size_t)nbs),
        v1v(3 * (size_t)nbs);
    for (int k = 0; k < nbs; ++k) mv[k] = val(mbs[k]);
    std::vector<Event> stat;
    do {
        const double tmp0 = std::fabs(h0) - std::fabs(tlocal);
        hrec = hlocal;
        if (std::fabs(hlocal) > tmp0) hlocal = std::copysign(tmp0, h0);
        x0 = xbs;
        v0 = vbs;
        double hdid = 0.0;
        if (mdt_bs2_with(force, tlocal, hlocal, hdid, tol, nbs, xbs.data(), vbs.data(), nullptr)) return 1;
        tlocal = tlocal + hdid;
        const double temp = time + tlocal;
        for (size_t k = 0; k < 3 * (size_t)nbs; ++k) {
            x0v[k] = val(x0[k]);
            v0v[k] = val(v0[k]);
            x1v[k] = val(xbs[k]);
            v1v[k] = val(vbs[k]);
        }
        stat.clear();
        mce_stat<double>(temp, hdid, nbs, nbsbig, mv.data(), x0v.data(), v0v.data(), x1v.data(), v1v.data(),
                         rcebs.data(), rphybs.data(), stat);
        for (Event e : stat) {
            e.i = index[e.i - 1] + 1;
            e.j = index[e.j - 1] + 1;
            events.push_back(e);
        }
    } while ((tlocal - h0) * h0 < 0.0);
    for (int k = 1; k < nbs; ++k) {
        const int j = index[k];
        for (int c = 0; c < 3; ++c) {
            x[3 * j + c] = xbs[3 * k + c];
            v[3 * j + c] = vbs[3 * k + c];
        }
    }
    return 0;
}

// mdt_hy, mercury6_2.for:3618-3782 (the CPU branch): democratic-heliocentric
// x, v in place; events receive the encounter records of mdt_hkce; *nce the
// number of encounter pairs of the step. Any scalar type R: mce_snif and the
// step control of the encounter subsystem read the values.
template <class R>
int mdt_hy(double time, double h0, double tol, const double* jcen, int nbod, int nbig, const R* m, R* x, R* v,
           const R* ngf, int ngflag, const double* rphys, const double* rcrit, const double* rce, HyState<R>& st,
           std::vector<Event>& events, int* nce_out, long long* forces) {
    const double hby2 = h0 * 0.5;
    const size_t nv = 3 * (size_t)nbod;
    if (st.a.size() < nv) {
        st.a.assign(nv, R(0.0));
        st.angf.assign(nv, R(0.0));
    }
    R* a = st.a.data();
    R* angf = st.angf.data();
    if (st.dtflag != 2) {
        if (st.dtflag == 0) st.hrec = h0;
        mfo_hy(jcen, nbod, nbig, m, x, rcrit, a);
        if (forces) ++*forces;
        st.dtflag = 2;
        for (size_t k = 3; k < nv; ++k) angf[k] = R(0.0);
        if (ngflag == 1 || ngflag == 3)
            if (mfo_ngf(nbod, x, v, angf, ngf)) return 1;
    }
    const R ausr = R(0.0);
    for (size_t k = 3; k < nv; ++k) v[k] = v[k] + R(hby2) * (angf[k] + ausr + a[k]);
    solar_drift(nbod, m, x, v, hby2);
    std::vector<R> x0(x, x + nv), v0(v, v + nv);
    for (int j = 1; j < nbod; ++j) {
        int iflag = 0;
        drift_one<R>(m[0], x[3 * j], x[3 * j + 1], x[3 * j + 2], v[3 * j], v[3 * j + 1], v[3 * j + 2], R(h0), iflag);
    }
    std::vector<double> x0v(nv), v0v(nv), x1v(nv), v1v(nv);
    for (size_t k = 0; k < nv; ++k) {
        x0v[k] = val(x0[k]);
        v0v[k] = val(v0[k]);
        x1v[k] = val(x[k]);
        v1v[k] = val(v[k]);
    }
    std::vector<int> ce, ice, jce;
    mce_snif(h0, nbod, nbig, x0v.data(), v0v.data(), x1v.data(), v1v.data(), rcrit, ce, ice, jce);
    *nce_out = (int)ice.size();
    if (!ice.empty()) {
        for (int j = 1; j < nbod; ++j)
            if (ce[j] != 0)
                for (int c = 0; c < 3; ++c) {
                    x[3 * j + c] = x0[3 * j + c];
                    v[3 * j + c] = v0[3 * j + c];
                }
        if (mdt_hkce(time, h0, st.hrec, tol, nbod, nbig, m, x, v, rphys, rcrit, rce, ce, ice, jce, events, forces))
            return 1;
    }
    solar_drift(nbod, m, x, v, hby2);
    mfo_hy(jcen, nbod, nbig, m, x, rcrit, a);
    if (forces) ++*forces;
    if (ngflag == 1 || ngflag == 3)
        if (mfo_ngf(nbod, x, v, angf, ngf)) return 1;
    for (size_t k = 3; k < nv; ++k) v[k] = v[k] + R(hby2) * (angf[k] + ausr + a[k]);
    return 0;
}

}  // namespace oracle
