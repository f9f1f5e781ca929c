// Test infrastructure only: the C entry points of the CPU oracle, called through
// ctypes by tests/ and by bench.py's CPU-baseline leg. Arrays keep the Fortran
// layout of the reference host (x(3,n), ngf(5,n)); events use the layout of the
// reference's MercuryEvent (mercury_cuda.h:7-11).
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "oracle_mvs.hpp"
#include "oracle_ra15.hpp"
#include "oracle_bs.hpp"
#include "oracle_hy.hpp"
#include "oracle_dual.hpp"
#include "oracle_energy.hpp"
#include "oracle_io.hpp"

namespace oracle {
thread_local Tally tally;
}

using oracle::Counted;
using oracle::Event;
using oracle::MvsState;

namespace {

template <class R> std::vector<R> widen(const double* p, size_t n) {
    std::vector<R> out(n);
    for (size_t k = 0; k < n; ++k) out[k] = R(p[k]);
    return out;
}

bool event_less(const Event& a, const Event& b) {
    int ai = std::min(a.i, a.j), aj = std::max(a.i, a.j);
    int bi = std::min(b.i, b.j), bj = std::max(b.i, b.j);
    return ai < bi || (ai == bi && aj < bj);
}

struct StepEvent {
    int step;
    Event e;
};

}  // namespace

struct OracleRun {
    std::vector<StepEvent> events;
    int status = 0;
};

extern "C" {

// drift_one on one body; xv = {x, y, z, vx, vy, vz} updated in place.
// Returns drift_one's iflg.
int oracle_drift_one(double mu, double* xv, double dt) {
    int iflg = 0;
    oracle::drift_one<double>(mu, xv[0], xv[1], xv[2], xv[3], xv[4], xv[5], dt, iflg);
    return iflg;
}

// One mdt_mvs step (mercury6_2.for:3987-4101) over the whole system in place.
// acc/angf (3n each) and *dtflag carry mdt_mvs's saved state between calls.
// Pair events are written to ev (up to cap); *count receives the total.
int oracle_mvs_step(int n, int nbig, const double* m, double* x, double* v, const double* ngf,
                    int ngflag, const double* jcen, const double* rce, const double* rphys,
                    double time, double h, double* acc, double* angf, int* dtflag, Event* ev,
                    int cap, int* count) {
    MvsState<double> st;
    st.size(n);
    std::memcpy(st.a.data(), acc, sizeof(double) * 3 * n);
    std::memcpy(st.angf.data(), angf, sizeof(double) * 3 * n);
    st.dtflag = *dtflag;
    double minside = m[0];
    for (int j = 1; j < nbig; ++j) {
        double msofar = minside + m[j];
        st.gm[j] = m[0] * msofar / minside;
        minside = msofar;
    }
    std::vector<Event> events;
    int rc = oracle::mdt_mvs<double>(time, h, jcen, n, nbig, m, x, v, rce, rphys, ngf, ngflag, st, events);
    std::memcpy(acc, st.a.data(), sizeof(double) * 3 * n);
    std::memcpy(angf, st.angf.data(), sizeof(double) * 3 * n);
    *dtflag = st.dtflag;
    *count = (int)events.size();
    for (int k = 0; k < (int)events.size() && k < cap; ++k) ev[k] = events[k];
    return rc;
}

// mce_cent over bodies 2..n (mercury6_2.for:1059-1167).
int oracle_mce_cent(int n, const double* m, const double* x0, const double* v0, const double* x1,
                    const double* v1, double time, double h, double rcen, Event* ev, int cap,
                    int* count) {
    std::vector<Event> events;
    oracle::mce_cent<double>(time, h, rcen, 1, n, m, x0, v0, x1, v1, events);
    *count = (int)events.size();
    for (int k = 0; k < (int)events.size() && k < cap; ++k) ev[k] = events[k];
    return 0;
}

// Output corrector: forward != 0 is mco_mvs2h, forward == 0 is mco_h2mvs.
int oracle_mvs_corrector(int forward, int n, int nbig, const double* m, const double* x,
                         const double* v, const double* ngf, int ngflag, const double* jcen,
                         double h, double* xh, double* vh) {
    return oracle::mvs_corrector<double>(forward != 0, h, jcen, n, nbig, m, x, v, ngf, ngflag, xh, vh);
}

// mce_hill (mercury6_2.for:1285-1314): Hill radii and semi-major axes.
void oracle_mce_hill(int n, const double* m, const double* x, const double* v, double* hill,
                     double* a) {
    oracle::mce_hill<double>(n, m, x, v, hill, a);
}

void oracle_mce_init(double h, double cefac, int n, const double* m, const double* x, const double* v,
                     const double* rho, const double* rceh, double* rphys, double* rce, double* rcrit,
                     int rcritflag) {
    oracle::mce_init<double>(h, cefac, n, m, x, v, rho, rceh, rphys, rce, rcrit, rcritflag);
}

// The step loop of mal_hcon (mercury6_2.for:700-781) for MVS: nsteps calls of
// mdt_mvs, each followed (if central != 0) by mce_cent on the heliocentric
// states before and after the step; time advances by time = time + h.
// Particles are split into nthreads contiguous ranges; each thread integrates
// the Big bodies plus its range with the same statements, which gives the
// same bits as one pass over the whole system because massless bodies never
// act on anything in the MVS map. (Semi-active Small bodies with mass couple
// only through the central-body oblateness reaction; with jcen != 0 and such
// bodies present the run uses one thread.)
OracleRun* oracle_mvs_run(int n, int nbig, const double* m, double* x, double* v,
                          const double* ngf, int ngflag, const double* jcen, const double* rce,
                          const double* rphys, double time0, double h, int nsteps, double rcen,
                          int central, int nthreads) {
    OracleRun* run = new OracleRun();
    int nsmall = n - nbig;
    bool coupled = false;
    if (jcen[0] != 0.0 || jcen[1] != 0.0 || jcen[2] != 0.0)
        for (int j = nbig; j < n; ++j) coupled = coupled || m[j] != 0.0;
    if (nthreads < 1 || coupled) nthreads = 1;
    if (nthreads > nsmall) nthreads = std::max(1, nsmall);
    std::vector<std::vector<StepEvent>> per(nthreads);
    std::vector<int> status(nthreads, 0), lo(nthreads), hi(nthreads);
    struct Sub { std::vector<double> m, x, v, g, r, p; };
    std::vector<Sub> sub(nthreads);
    // Every thread's subsystem is gathered before any thread starts, and the
    // results are scattered back after all have joined.
    for (int t = 0; t < nthreads; ++t) {
        lo[t] = nbig + (int)((long long)nsmall * t / nthreads);
        hi[t] = nbig + (int)((long long)nsmall * (t + 1) / nthreads);
        int ns = nbig + (hi[t] - lo[t]);
        Sub& S = sub[t];
        S.m.resize(ns); S.x.resize(3 * ns); S.v.resize(3 * ns); S.g.resize(5 * ns);
        S.r.resize(ns); S.p.resize(ns);
        auto take = [&](int dst, int src) {
            S.m[dst] = m[src]; S.r[dst] = rce[src]; S.p[dst] = rphys[src];
            for (int c = 0; c < 3; ++c) { S.x[3 * dst + c] = x[3 * src + c]; S.v[3 * dst + c] = v[3 * src + c]; }
            for (int c = 0; c < 5; ++c) S.g[5 * dst + c] = ngf[5 * src + c];
        };
        for (int k = 0; k < nbig; ++k) take(k, k);
        for (int k = lo[t]; k < hi[t]; ++k) take(nbig + (k - lo[t]), k);
    }
    auto work = [&](int t) {
        Sub& S = sub[t];
        int ns = (int)S.m.size();
        int offset = lo[t] - nbig;
        MvsState<double> st;
        st.size(ns);
        std::vector<double> xh0(3 * ns), vh0(3 * ns);
        std::vector<Event> events;
        double time = time0;
        for (int s = 0; s < nsteps; ++s) {
            std::copy(S.x.begin(), S.x.end(), xh0.begin());
            std::copy(S.v.begin(), S.v.end(), vh0.begin());
            events.clear();
            if (oracle::mdt_mvs<double>(time, h, jcen, ns, nbig, S.m.data(), S.x.data(), S.v.data(),
                                        S.r.data(), S.p.data(), S.g.data(), ngflag, st, events)) {
                status[t] = 1;
                return;
            }
            time = time + h;
            if (central)
                oracle::mce_cent<double>(time, h, rcen, 1, ns, S.m.data(), xh0.data(), vh0.data(),
                                         S.x.data(), S.v.data(), events);
            for (Event e : events) {
                bool big_only = e.i <= nbig && e.j <= nbig;
                if (big_only && t != 0) continue;
                if (e.i > nbig) e.i += offset;
                if (e.j > nbig) e.j += offset;
                per[t].push_back(StepEvent{s, e});
            }
        }
    };
    if (nthreads == 1) work(0);
    else {
        std::vector<std::thread> pool;
        for (int t = 0; t < nthreads; ++t) pool.emplace_back(work, t);
        for (auto& th : pool) th.join();
    }
    for (int t = 0; t < nthreads; ++t) {
        const Sub& S = sub[t];
        if (t == 0)
            for (int k = 0; k < 3 * nbig; ++k) { x[k] = S.x[k]; v[k] = S.v[k]; }
        for (int k = lo[t]; k < hi[t]; ++k)
            for (int c = 0; c < 3; ++c) {
                x[3 * k + c] = S.x[3 * (nbig + k - lo[t]) + c];
                v[3 * k + c] = S.v[3 * (nbig + k - lo[t]) + c];
            }
    }
    for (int t = 0; t < nthreads; ++t) {
        run->status |= status[t];
        run->events.insert(run->events.end(), per[t].begin(), per[t].end());
    }
    std::stable_sort(run->events.begin(), run->events.end(), [](const StepEvent& a, const StepEvent& b) {
        if (a.step != b.step) return a.step < b.step;
        return event_less(a.e, b.e);
    });
    return run;
}

int oracle_run_status(const OracleRun* run) { return run->status; }
int oracle_run_event_count(const OracleRun* run) { return (int)run->events.size(); }
void oracle_run_events(const OracleRun* run, Event* dst, int* steps) {
    for (size_t k = 0; k < run->events.size(); ++k) {
        dst[k] = run->events[k].e;
        if (steps) steps[k] = run->events[k].step;
    }
}
void oracle_run_free(OracleRun* run) { delete run; }

// Algorithmic operation tally of nsteps MVS steps (mdt_mvs + mce_cent) of the
// given system: out = {add, mul, div, sqrt, cmp, libm}. The state is not
// modified. Each +,- counts as add, * as mul, / as div.
void oracle_count_mvs(int n, int nbig, const double* m, const double* x, const double* v,
                      const double* ngf, int ngflag, const double* jcen, const double* rce,
                      const double* rphys, double time0, double h, int nsteps, double rcen,
                      uint64_t* out) {
    auto cm = widen<Counted>(m, n), cx = widen<Counted>(x, 3 * n), cv = widen<Counted>(v, 3 * n);
    auto cg = widen<Counted>(ngf, 5 * n), cr = widen<Counted>(rce, n), cp = widen<Counted>(rphys, n);
    MvsState<Counted> st;
    st.size(n);
    std::vector<Counted> xh0(3 * n), vh0(3 * n);
    std::vector<Event> events;
    oracle::tally = oracle::Tally();
    Counted time = time0;
    for (int s = 0; s < nsteps; ++s) {
        xh0 = cx;
        vh0 = cv;
        events.clear();
        oracle::mdt_mvs<Counted>(time, Counted(h), jcen, n, nbig, cm.data(), cx.data(), cv.data(),
                                 cr.data(), cp.data(), cg.data(), ngflag, st, events);
        time = Counted(time.v + h);
        oracle::mce_cent<Counted>(time, Counted(h), Counted(rcen), 1, n, cm.data(), xh0.data(),
                                  vh0.data(), cx.data(), cv.data(), events);
    }
    out[0] = oracle::tally.add;
    out[1] = oracle::tally.mul;
    out[2] = oracle::tally.div;
    out[3] = oracle::tally.sqrt;
    out[4] = oracle::tally.cmp;
    out[5] = oracle::tally.libm;
}

// Single force laws for known-answer tests: 0 = mfo_pr, 1 = mfo_ngf, 2 = mfo_pn.
int oracle_force_term(int which, int n, const double* m, const double* x, const double* v, const double* ngf,
                      double* a) {
    if (which == 0) oracle::mfo_pr<double>(n, m, x, v, a, ngf);
    else if (which == 1) return oracle::mfo_ngf<double>(n, x, v, a, ngf);
    else oracle::mfo_pn<double>(n, m, x, v, a);
    return 0;
}

// mfo_all (mercury6_2.for:4506-4571) on the whole system; a(3n) out.
int oracle_force(int n, int nbig, const double* m, const double* x, const double* v, const double* ngf,
                 int ngflag, int pn, const double* jcen, double* a) {
    return oracle::mfo_all<double>(jcen, n, nbig, m, x, v, a, ngf, ngflag, pn);
}

// Variable-step RA15 loop in the manner of mal_hvar (mercury6_2.for:389-463)
// from time0 towards tstop: each step is clipped to the remaining interval
// (clipped_step, mercury_support.f90:207-212), a clipped step restarts the
// predictor (dtflag = 1, mercury6_2.for:429), and after each step mce_stat
// (x0,v0 = the state before the step) and, if central != 0, mce_cent screen
// for events. h is the initial trial step (in/out). Returns the number of
// steps, or -1 on failure; events are kept in the run handle.
// mal_hvar's step loop (mercury6_2.for:423-470) with algor 2 (mdt_bs1),
// 3 (mdt_bs2) or 4 (mdt_ra15): steps clipped to tstop (a clipped RA15 step
// restarts the sequence), then mce_stat and mce_cent on the step. *h is the
// trial step in, the next one out; counters = {steps, force calls, rejected}.
OracleRun* oracle_hvar_run(int algor, int n, int nbig, const double* m, double* x, double* v, const double* ngf,
                           int ngflag, int pn, const double* jcen, const double* rce, const double* rphys,
                           double time0, double tstop, double* h, double tol, double rcen, int central,
                           int max_steps, long long* counters) {
    OracleRun* run = new OracleRun();
    oracle::Ra15State st;
    st.size(n);
    std::vector<double> x0(3 * n), v0(3 * n);
    double time = time0;
    long long forces = 0, steps = 0, rejected = 0;
    std::vector<Event> events;
    while (steps < max_steps) {
        if (std::fabs(tstop - time) <= 0.0) break;
        double target = tstop;
        double step = std::copysign(std::min(std::fabs(target - time), std::fabs(*h)), target - time);
        if (!std::isfinite(step) || time + step == time) break;
        if (algor == 4 && step != *h && st.dtflag != 0) st.dtflag = 1;
        *h = step;
        std::copy(x, x + 3 * n, x0.begin());
        std::copy(v, v + 3 * n, v0.begin());
        double hdid = 0.0;
        int rc;
        if (algor == 2)
            rc = oracle::mdt_bs1(time, *h, hdid, tol, jcen, n, nbig, m, x, v, ngf, ngflag, pn, &forces, &rejected);
        else if (algor == 3)
            rc = oracle::mdt_bs2(time, *h, hdid, tol, jcen, n, nbig, m, x, v, ngf, ngflag, pn, &forces, &rejected);
        else
            rc = oracle::mdt_ra15(time, *h, hdid, tol, jcen, n, nbig, m, x, v, ngf, ngflag, pn, st, &forces);
        if (rc) {
            run->status = 1;
            break;
        }
        time = time + hdid;
        events.clear();
        oracle::mce_stat<double>(time, hdid, n, nbig, m, x0.data(), v0.data(), x, v, rce, rphys, events);
        if (central) oracle::mce_cent<double>(time, hdid, rcen, 1, n, m, x0.data(), v0.data(), x, v, events);
        std::stable_sort(events.begin(), events.end(), event_less);
        for (auto& e : events) run->events.push_back(StepEvent{(int)steps, e});
        ++steps;
    }
    if (counters) {
        counters[0] = steps;
        counters[1] = forces;
        counters[2] = rejected;
    }
    return run;
}

// mal_hcon's loop with algor 10 (mdt_hy, mercury6_2.for:3618-3782) on the
// democratic-heliocentric state (x, v in place): per step the encounter
// records of mdt_hkce, then mce_cent on the heliocentric (mco_dh2h) states
// before and after the step. counters = {force calls, encounter pairs}.
OracleRun* oracle_hy_run(int n, int nbig, const double* m, double* x, double* v, const double* ngf, int ngflag,
                         const double* jcen, const double* rce, const double* rphys, const double* rcrit,
                         double time0, double h, int nsteps, double tol, double rcen, int central,
                         long long* counters) {
    OracleRun* run = new OracleRun();
    oracle::HyState<double> st;
    std::vector<double> xh0(3 * n), vh0(3 * n), vh1(3 * n);
    long long forces = 0, pairs = 0;
    double time = time0;
    std::vector<Event> events;
    for (int s = 0; s < nsteps; ++s) {
        std::copy(x, x + 3 * n, xh0.begin());
        oracle::dh2h_velocity(n, m, v, vh0.data());
        events.clear();
        int nce = 0;
        if (oracle::mdt_hy(time, h, tol, jcen, n, nbig, m, x, v, ngf, ngflag, rphys, rcrit, rce, st, events, &nce,
                           &forces)) {
            run->status = 1;
            break;
        }
        pairs += nce;
        time = time + h;
        if (central) {
            oracle::dh2h_velocity(n, m, v, vh1.data());
            oracle::mce_cent<double>(time, h, rcen, 1, n, m, xh0.data(), vh0.data(), x, vh1.data(), events);
        }
        std::stable_sort(events.begin(), events.end(), event_less);
        for (auto& e : events) run->events.push_back(StepEvent{s, e});
    }
    if (counters) {
        counters[0] = forces;
        counters[1] = pairs;
    }
    return run;
}

// mce_snif on given states (0-based pairs into ice/jce, up to cap); returns
// the pair count.
int oracle_mce_snif(double h, int n, int nbig, const double* x0, const double* v0, const double* x1,
                    const double* v1, const double* rcrit, int* ice, int* jce, int cap) {
    std::vector<int> ce, vi, vj;
    oracle::mce_snif(h, n, nbig, x0, v0, x1, v1, rcrit, ce, vi, vj);
    for (size_t k = 0; k < vi.size() && (int)k < cap; ++k) {
        ice[k] = vi[k];
        jce[k] = vj[k];
    }
    return (int)vi.size();
}

// mfo_hy of the whole system into a (n, 3).
void oracle_mfo_hy(int n, int nbig, const double* m, const double* x, const double* rcrit, const double* jcen,
                   double* a) {
    oracle::mfo_hy(jcen, n, nbig, m, x, rcrit, a);
}

// drift_one of one body with its 6x6 Jacobian (row-major, d out / d in) by
// forward-mode dual numbers; xv = {x, y, z, vx, vy, vz} updated in place.
void oracle_drift_jacobian(double mu, double* xv, double dt, double* jac) {
    using D6 = oracle::Dual<6>;
    D6 q[6];
    for (int c = 0; c < 6; ++c) {
        q[c] = D6(xv[c]);
        q[c].d[c] = 1.0;
    }
    int iflg = 0;
    oracle::drift_one<D6>(D6(mu), q[0], q[1], q[2], q[3], q[4], q[5], D6(dt), iflg);
    for (int c = 0; c < 6; ++c) {
        xv[c] = q[c].v;
        for (int k = 0; k < 6; ++k) jac[6 * c + k] = q[c].d[k];
    }
}

// nsteps of mdt_mvs (no central screen needed: states only) with the
// derivatives of every massless particle's final state with respect to its
// own initial position, velocity and Yarkovsky coefficient ngf(5,j), by
// forward-mode dual numbers through the same statements. jac receives, per
// particle (bodies nbig..n-1 in order), a 6x7 matrix row-major: rows x,y,z,
// vx,vy,vz at the end; columns x0,y0,z0,vx0,vy0,vz0,yar. x, v are advanced in
// place. Returns nonzero on a force failure or a massive Small body.
int oracle_mvs_jacobian(int n, int nbig, const double* m, double* x, double* v, const double* ngf, int ngflag,
                        const double* jcen, double h, int nsteps, double* jac) {
    using DD = oracle::Dual<7>;
    for (int j = nbig; j < n; ++j)
        if (m[j] != 0.0) return 1;
    std::vector<DD> dm(n), dx(3 * (size_t)n), dv(3 * (size_t)n), dngf(5 * (size_t)n), drce(n, DD(0.0)),
        drph(n, DD(0.0));
    for (int j = 0; j < n; ++j) {
        dm[j] = DD(m[j]);
        for (int c = 0; c < 3; ++c) {
            dx[3 * j + c] = DD(x[3 * j + c]);
            dv[3 * j + c] = DD(v[3 * j + c]);
            if (j >= nbig) {
                dx[3 * j + c].d[c] = 1.0;
                dv[3 * j + c].d[3 + c] = 1.0;
            }
        }
        for (int c = 0; c < 5; ++c) dngf[5 * j + c] = DD(ngf[5 * j + c]);
        if (j >= nbig) dngf[5 * j + 4].d[6] = 1.0;
    }
    oracle::MvsState<DD> st;
    std::vector<Event> events;
    DD time(0.0), hh(h);
    for (int s = 0; s < nsteps; ++s) {
        events.clear();
        if (oracle::mdt_mvs<DD>(time, hh, jcen, n, nbig, dm.data(), dx.data(), dv.data(), drce.data(), drph.data(),
                                dngf.data(), ngflag, st, events))
            return 1;
        time = time + hh;
    }
    for (int j = 0; j < n; ++j)
        for (int c = 0; c < 3; ++c) {
            x[3 * j + c] = dx[3 * j + c].v;
            v[3 * j + c] = dv[3 * j + c].v;
        }
    for (int j = nbig; j < n; ++j) {
        double* J = jac + 42 * (size_t)(j - nbig);
        for (int c = 0; c < 3; ++c)
            for (int k = 0; k < 7; ++k) {
                J[7 * c + k] = dx[3 * j + c].d[k];
                J[7 * (3 + c) + k] = dv[3 * j + c].d[k];
            }
    }
    return 0;
}

// nsteps of mdt_hy (democratic-heliocentric x, v in place) with the
// derivatives of every massless particle's final state with respect to its own
// initial position, velocity and Yarkovsky coefficient ngf(5,j), by
// forward-mode dual numbers through the same statements: the kicks with the
// changeover force, the solar drifts, the Kepler drift and, for the steps in
// which a particle is an encounter member, mdt_hkce's BS2 integration with the
// substep sequence its step control chooses (decisions read the values).
// jac as for oracle_mvs_jacobian (6x7 per particle, row-major). Returns
// nonzero on a failure or a massive Small body.
int oracle_hy_jacobian(int n, int nbig, const double* m, double* x, double* v, const double* ngf, int ngflag,
                       const double* rcrit, double h, int nsteps, double tol, double* jac) {
    using DD = oracle::Dual<7>;
    for (int j = nbig; j < n; ++j)
        if (m[j] != 0.0) return 1;
    std::vector<DD> dm(n), dx(3 * (size_t)n), dv(3 * (size_t)n), dngf(5 * (size_t)n);
    for (int j = 0; j < n; ++j) {
        dm[j] = DD(m[j]);
        for (int c = 0; c < 3; ++c) {
            dx[3 * j + c] = DD(x[3 * j + c]);
            dv[3 * j + c] = DD(v[3 * j + c]);
            if (j >= nbig) {
                dx[3 * j + c].d[c] = 1.0;
                dv[3 * j + c].d[3 + c] = 1.0;
            }
        }
        for (int c = 0; c < 5; ++c) dngf[5 * j + c] = DD(ngf[5 * j + c]);
        if (j >= nbig) dngf[5 * j + 4].d[6] = 1.0;
    }
    const double jcen[3] = {0.0, 0.0, 0.0};
    std::vector<double> zeros(n, 0.0);
    oracle::HyState<DD> st;
    std::vector<Event> events;
    double time = 0.0;
    for (int s = 0; s < nsteps; ++s) {
        events.clear();
        int nce = 0;
        if (oracle::mdt_hy<DD>(time, h, tol, jcen, n, nbig, dm.data(), dx.data(), dv.data(), dngf.data(), ngflag,
                               zeros.data(), rcrit, zeros.data(), st, events, &nce, nullptr))
            return 1;
        time = time + h;
    }
    for (int j = 0; j < n; ++j)
        for (int c = 0; c < 3; ++c) {
            x[3 * j + c] = dx[3 * j + c].v;
            v[3 * j + c] = dv[3 * j + c].v;
        }
    for (int j = nbig; j < n; ++j) {
        double* J = jac + 42 * (size_t)(j - nbig);
        for (int c = 0; c < 3; ++c)
            for (int k = 0; k < 7; ++k) {
                J[7 * c + k] = dx[3 * j + c].d[k];
                J[7 * (3 + c) + k] = dv[3 * j + c].d[k];
            }
    }
    return 0;
}

// mxx_ejec's test (mercury6_2.for:7071-7082): the 1-based ids (ascending) of
// bodies j >= i0 (1-based; i0 <= 0 means 2) with x*x + y*y + z*z > rmax^2.
int oracle_mxx_ejec(int n, int i0, const double* x, double rmax, int* ids) {
    if (i0 <= 0) i0 = 2;
    const double rmax2 = rmax * rmax;
    int k = 0;
    for (int j = i0; j <= n; ++j) {
        const double* p = x + 3 * (size_t)(j - 1);
        const double r2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
        if (r2 > rmax2) ids[k++] = j;
    }
    return k;
}

// mio_ce's record bodies (70 characters each) of the close encounters
// (kind bit 1) among n event records, in order; returns their count.
int oracle_mio_ce(const Event* ev, int n, double mcen, double rcen, double rmax, unsigned char* lines) {
    int k = 0;
    for (int q = 0; q < n; ++q) {
        if (!(ev[q].kind & 1)) continue;
        oracle::mio_ce_record(ev[q].time, ev[q].i, ev[q].j, ev[q].distance, ev[q].xi, ev[q].xj, mcen, rcen, rmax,
                              lines + 70 * (size_t)k);
        ++k;
    }
    return k;
}

// mxx_sync's ordering (mercury6_2.for:7468-7486 with mxx_sort, 7392-7421):
// Small bodies by epoch (Shell sort, gaps 1, 4, 13, ...), reversed when the
// last is further from tstart than the first. order[k] = the 0-based Small
// body at position k.
int oracle_epoch_order(int nsml, const double* epochs, double tstart, int* order) {
    std::vector<double> epsml(epochs, epochs + nsml);
    std::vector<int> indx(nsml);
    for (int i = 1; i <= nsml; ++i) indx[i - 1] = i;
    int inc = 1;
    while (inc < nsml / 3) inc = 3 * inc + 1;
    while (inc >= 1) {
        for (int i = inc + 1; i <= nsml; ++i) {
            const double y = epsml[i - 1];
            const int iy = indx[i - 1];
            int j = i;
            while (j > inc) {
                if (epsml[j - inc - 1] <= y) break;
                epsml[j - 1] = epsml[j - inc - 1];
                indx[j - 1] = indx[j - inc - 1];
                j = j - inc;
            }
            epsml[j - 1] = y;
            indx[j - 1] = iy;
        }
        inc = inc / 3;
    }
    if (nsml > 0 && std::fabs(epsml[0] - tstart) < std::fabs(epsml[nsml - 1] - tstart)) {
        const int k = nsml + 1;
        for (int j = 1; j <= nsml / 2; ++j) {
            const int l = k - j;
            std::swap(epsml[j - 1], epsml[l - 1]);
            std::swap(indx[j - 1], indx[l - 1]);
        }
    }
    for (int i = 0; i < nsml; ++i) order[i] = indx[i] - 1;
    return 0;
}

// mxx_sync's integration (mercury6_2.for:7556-7570) on bodies already in its
// order: for each Small body j, the bodies before it are advanced by mdt_bs1
// to j's epoch (steps clipped by mercury_support.f90:207-212, epochs matched
// within 202-205). *time: in the Big bodies' epoch, out the last epoch.
// Returns nonzero on a failure; *steps counts the BS steps.
int oracle_mxx_sync(int n, int nbig, const double* m, double* x, double* v, const double* ngf, int ngflag, int pn,
                    const double* jcen, const double* epoch, double* time, double h0, double tol, double dtout,
                    int* steps) {
    auto spacing = [](double a) {
        a = std::fabs(a);
        if (a == 0.0) return 2.2250738585072014e-308;
        int e = 0;
        std::frexp(a, &e);
        return std::ldexp(1.0, e - 53);
    };
    auto eps = [&](double t, double target) {
        return std::max(1e-13, 2.0 * spacing(std::max(std::fabs(t), std::fabs(target))));
    };
    double t = *time, h = h0;
    int count = 0;
    for (int j = nbig + 1; j <= n; ++j) {
        const int nsofar = j - 1;
        while (std::fabs(t - epoch[j - 1]) > eps(t, epoch[j - 1])) {
            const double target = epoch[j - 1];
            const double step = std::copysign(
                std::min(std::min(std::fabs(target - t), std::fabs(h)), std::fabs(dtout)), target - t);
            if (!std::isfinite(step) || t + step == t) return 1;
            h = step;
            double hdid = 0.0;
            if (oracle::mdt_bs1(t, h, hdid, tol, jcen, nsofar, nbig, m, x, v, ngf, ngflag, pn, nullptr, nullptr))
                return 1;
            t = t + hdid;
            ++count;
        }
    }
    *time = t;
    *steps = count;
    return 0;
}

// mxx_en of n bodies (Fortran layout); s may be null. out = {e, l2}.
void oracle_mxx_en(int n, const double* m, const double* xh, const double* vh, const double* s, const double* jcen,
                   double* out) {
    oracle::mxx_en<double>(jcen, n, m, xh, vh, s, out[0], out[1]);
}

}  // extern "C"
