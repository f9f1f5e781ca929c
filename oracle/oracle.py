"""Test infrastructure only: ctypes front end of the CPU oracle.

The oracle (``oracle_mvs.hpp`` and friends, built into ``liboracle.so``) is a
statement-for-statement C++ restatement of MERCURY6's Fortran hot path
(mercury6_2.for). It is the parity checker for the CUDA library: only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may load it, and
never as the thing measured or shipped.

Arrays follow the reference host's Fortran layout: ``x`` is (n, 3) row-major,
which is byte-identical to Fortran's x(3,n); ``ngf`` is (n, 5).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_KEPLER = HERE / "_ref" / "libkepler_ref.so"
REF_CUDA = HERE / "_ref" / "libmercury_cuda_ref.so"

D = C.c_double
I = C.c_int
PD = C.POINTER(C.c_double)


class Event(C.Structure):
    """Layout of the reference's MercuryEvent (mercury_cuda.h:7-11)."""

    _fields_ = [("i", C.c_int), ("j", C.c_int), ("kind", C.c_int), ("now", C.c_int),
                ("distance", C.c_double), ("time", C.c_double),
                ("xi", C.c_double * 6), ("xj", C.c_double * 6)]


EVENT_DTYPE = np.dtype([("i", np.int32), ("j", np.int32), ("kind", np.int32), ("now", np.int32),
                        ("distance", np.float64), ("time", np.float64),
                        ("xi", np.float64, 6), ("xj", np.float64, 6)])
assert EVENT_DTYPE.itemsize == C.sizeof(Event) == 128


def build() -> None:
    """Compile liboracle.so with the Makefile beside this file (g++ only)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        L.oracle_drift_one.argtypes = [D, PD, D]
        L.oracle_drift_one.restype = I
        L.oracle_mvs_step.argtypes = [I, I, PD, PD, PD, PD, I, PD, PD, PD, D, D, PD, PD,
                                      C.POINTER(I), C.c_void_p, I, C.POINTER(I)]
        L.oracle_mvs_step.restype = I
        L.oracle_mce_cent.argtypes = [I, PD, PD, PD, PD, PD, D, D, D, C.c_void_p, I, C.POINTER(I)]
        L.oracle_mvs_corrector.argtypes = [I, I, I, PD, PD, PD, PD, I, PD, D, PD, PD]
        L.oracle_mvs_corrector.restype = I
        L.oracle_mce_hill.argtypes = [I, PD, PD, PD, PD, PD]
        L.oracle_mce_init.argtypes = [D, D, I, PD, PD, PD, PD, PD, PD, PD, PD, I]
        L.oracle_mce_init.restype = None
        L.oracle_mvs_run.argtypes = [I, I, PD, PD, PD, PD, I, PD, PD, PD, D, D, I, D, I, I]
        L.oracle_mvs_run.restype = C.c_void_p
        L.oracle_run_status.argtypes = [C.c_void_p]
        L.oracle_run_event_count.argtypes = [C.c_void_p]
        L.oracle_run_events.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_run_free.argtypes = [C.c_void_p]
        L.oracle_count_mvs.argtypes = [I, I, PD, PD, PD, PD, I, PD, PD, PD, D, D, I, D,
                                       C.POINTER(C.c_uint64)]
        L.oracle_force.argtypes = [I, I, PD, PD, PD, PD, I, I, PD, PD]
        L.oracle_force.restype = I
        L.oracle_force_term.argtypes = [I, I, PD, PD, PD, PD, PD]
        L.oracle_force_term.restype = I
        L.oracle_hvar_run.argtypes = [I, I, I, PD, PD, PD, PD, I, I, PD, PD, PD, D, D, PD, D, D, I, I,
                                      C.POINTER(C.c_longlong)]
        L.oracle_hvar_run.restype = C.c_void_p
        L.oracle_hy_run.argtypes = [I, I, PD, PD, PD, PD, I, PD, PD, PD, PD, D, D, I, D, D, I,
                                    C.POINTER(C.c_longlong)]
        L.oracle_hy_run.restype = C.c_void_p
        PI_ = C.POINTER(I)
        L.oracle_mce_snif.argtypes = [D, I, I, PD, PD, PD, PD, PD, PI_, PI_, I]
        L.oracle_mce_snif.restype = I
        L.oracle_mfo_hy.argtypes = [I, I, PD, PD, PD, PD, PD]
        L.oracle_mvs_jacobian.argtypes = [I, I, PD, PD, PD, PD, I, PD, D, I, PD]
        L.oracle_mvs_jacobian.restype = I
        L.oracle_hy_jacobian.argtypes = [I, I, PD, PD, PD, PD, I, PD, D, I, D, PD]
        L.oracle_hy_jacobian.restype = I
        L.oracle_mxx_ejec.argtypes = [I, I, PD, D, C.POINTER(I)]
        L.oracle_mxx_ejec.restype = I
        L.oracle_mio_ce.argtypes = [C.c_void_p, I, D, D, D, C.c_void_p]
        L.oracle_mio_ce.restype = I
        L.oracle_epoch_order.argtypes = [I, PD, D, C.POINTER(I)]
        L.oracle_epoch_order.restype = I
        L.oracle_mxx_sync.argtypes = [I, I, PD, PD, PD, PD, I, I, PD, PD, PD, D, D, D, C.POINTER(I)]
        L.oracle_mxx_sync.restype = I
        L.oracle_mxx_en.argtypes = [I, PD, PD, PD, C.c_void_p, PD, PD]
        L.oracle_mxx_en.restype = None
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(PD)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def drift_one(mu: float, xv, dt: float):
    """drift_one (mercury6_2.for:8296-8330) on one 6-vector; returns (xv', iflg)."""
    s = _f64(xv).copy()
    flag = lib().oracle_drift_one(mu, _p(s), dt)
    return s, flag


def ref_drift_one(mu: float, xv, dt: float):
    """The reference's own drift_one__ (mercury_cuda_kepler.cuh) built for the host."""
    L = C.CDLL(str(REF_KEPLER))
    L.ref_drift_one.argtypes = [D, PD, D]
    L.ref_drift_one.restype = I
    s = _f64(xv).copy()
    flag = L.ref_drift_one(mu, _p(s), dt)
    return s, flag


class MvsStepper:
    """mdt_mvs with its saved state (cached accelerations, dtflag) held here."""

    def __init__(self, sys):
        self.sys = sys
        n = sys.n
        self.acc = np.zeros((n, 3))
        self.angf = np.zeros((n, 3))
        self.dtflag = I(0)

    def step(self, time: float, h: float):
        s = self.sys
        cap = max(64, s.n)
        buf = np.zeros(cap, dtype=EVENT_DTYPE)
        count = I(0)
        rc = lib().oracle_mvs_step(s.n, s.nbig, _p(s.m), _p(s.x), _p(s.v), _p(s.ngf), s.ngflag,
                                   _p(s.jcen), _p(s.rce), _p(s.rphys), time, h, _p(self.acc),
                                   _p(self.angf), C.byref(self.dtflag),
                                   buf.ctypes.data_as(C.c_void_p), cap, C.byref(count))
        if rc:
            raise RuntimeError("oracle mdt_mvs failed (mfo_ngf undefined direction)")
        assert count.value <= cap
        return buf[:count.value].copy()


def mce_cent(m, x0, v0, x1, v1, time, h, rcen):
    n = len(m)
    cap = max(16, n)
    buf = np.zeros(cap, dtype=EVENT_DTYPE)
    count = I(0)
    lib().oracle_mce_cent(n, _p(_f64(m)), _p(_f64(x0)), _p(_f64(v0)), _p(_f64(x1)), _p(_f64(v1)),
                          time, h, rcen, buf.ctypes.data_as(C.c_void_p), cap, C.byref(count))
    return buf[:count.value].copy()


def mvs_corrector(sys, h: float, forward: bool = True):
    """mco_mvs2h (forward) or mco_h2mvs (inverse) on copies of sys.x, sys.v."""
    xh = np.zeros_like(sys.x)
    vh = np.zeros_like(sys.v)
    rc = lib().oracle_mvs_corrector(int(forward), sys.n, sys.nbig, _p(sys.m), _p(sys.x), _p(sys.v),
                                    _p(sys.ngf), sys.ngflag, _p(sys.jcen), h, _p(xh), _p(vh))
    if rc:
        raise RuntimeError("oracle corrector failed")
    return xh, vh


def mce_hill(m, x, v):
    m = _f64(m)
    n = len(m)
    hill = np.zeros(n)
    a = np.zeros(n)
    lib().oracle_mce_hill(n, _p(m), _p(_f64(x)), _p(_f64(v)), _p(hill), _p(a))
    return hill, a


def mce_init(m, x, v, rho, rceh, h, cefac, rcritflag=1):
    """mce_init's limits (mercury6_2.for:1339-1380): (rce, rphys, rcrit); the
    central body's entries stay zero."""
    m, x, v, rho, rceh = map(_f64, (m, x, v, rho, rceh))
    n = len(m)
    rce, rphys, rcrit = np.zeros(n), np.zeros(n), np.zeros(n)
    lib().oracle_mce_init(float(h), float(cefac), n, _p(m), _p(x), _p(v), _p(rho), _p(rceh), _p(rphys), _p(rce),
                          _p(rcrit), int(rcritflag))
    return rce, rphys, rcrit


def mvs_run(sys, time0: float, h: float, nsteps: int, rcen: float, central: bool = True,
            threads: int | None = None):
    """mal_hcon's MVS step loop on sys (in place). Returns (events, steps)."""
    threads = threads or os.cpu_count() or 1
    s = sys
    handle = lib().oracle_mvs_run(s.n, s.nbig, _p(s.m), _p(s.x), _p(s.v), _p(s.ngf), s.ngflag,
                                  _p(s.jcen), _p(s.rce), _p(s.rphys), time0, h, nsteps, rcen,
                                  int(central), threads)
    try:
        if lib().oracle_run_status(handle):
            raise RuntimeError("oracle MVS run failed")
        count = lib().oracle_run_event_count(handle)
        events = np.zeros(count, dtype=EVENT_DTYPE)
        steps = np.zeros(count, dtype=np.int32)
        lib().oracle_run_events(handle, events.ctypes.data_as(C.c_void_p),
                                steps.ctypes.data_as(C.c_void_p))
    finally:
        lib().oracle_run_free(handle)
    return events, steps


def count_mvs(sys, time0: float, h: float, nsteps: int, rcen: float):
    """Algorithmic operation tally {add, mul, div, sqrt, cmp, libm} of nsteps steps."""
    s = sys
    out = (C.c_uint64 * 6)()
    lib().oracle_count_mvs(s.n, s.nbig, _p(s.m), _p(s.x), _p(s.v), _p(s.ngf), s.ngflag,
                           _p(s.jcen), _p(s.rce), _p(s.rphys), time0, h, nsteps, rcen, out)
    return dict(zip(["add", "mul", "div", "sqrt", "cmp", "libm"], list(out)))


def force(sys):
    """mfo_all (mercury6_2.for:4506-4571) of the whole system, shape (n, 3)."""
    a = np.zeros((sys.n, 3))
    rc = lib().oracle_force(sys.n, sys.nbig, _p(sys.m), _p(sys.x), _p(sys.v), _p(sys.ngf), sys.ngflag,
                            int(sys.pn), _p(sys.jcen), _p(a))
    if rc:
        raise RuntimeError("oracle mfo_all failed")
    return a


def force_term(which, m, x, v, ngf):
    """One force law alone: 'pr' (mfo_pr), 'ngf' (mfo_ngf) or 'pn' (mfo_pn)."""
    code = {"pr": 0, "ngf": 1, "pn": 2}[which]
    m, x, v, ngf = _f64(m), _f64(x), _f64(v), _f64(ngf)
    a = np.zeros_like(x)
    if lib().oracle_force_term(code, len(m), _p(m), _p(x), _p(v), _p(ngf), _p(a)):
        raise RuntimeError("oracle force law failed")
    return a


def hvar_run(sys, algorithm, time0, tstop, h, tol, rcen=0.005, central=True, max_steps=1_000_000):
    """mal_hvar's loop with mdt_bs1 (2), mdt_bs2 (3) or mdt_ra15 (4) on sys (in place).

    Returns (events, step of each event, h_next, steps, force calls, rejected)."""
    s = sys
    hh = D(h)
    counters = (C.c_longlong * 3)()
    handle = lib().oracle_hvar_run(int(algorithm), s.n, s.nbig, _p(s.m), _p(s.x), _p(s.v), _p(s.ngf), s.ngflag,
                                   int(s.pn), _p(s.jcen), _p(s.rce), _p(s.rphys), time0, tstop, C.byref(hh), tol,
                                   rcen, int(central), int(max_steps), counters)
    try:
        if lib().oracle_run_status(handle):
            raise RuntimeError("oracle integration failed")
        count = lib().oracle_run_event_count(handle)
        events = np.zeros(count, dtype=EVENT_DTYPE)
        steps = np.zeros(count, dtype=np.int32)
        lib().oracle_run_events(handle, events.ctypes.data_as(C.c_void_p), steps.ctypes.data_as(C.c_void_p))
    finally:
        lib().oracle_run_free(handle)
    return events, steps, hh.value, counters[0], counters[1], counters[2]


def ra15_run(sys, time0, tstop, h, tol, rcen=0.005, central=True, max_steps=1_000_000):
    """mal_hvar-style RA15 loop on sys (in place). Returns (events, steps, h_next, nsteps, nforces)."""
    ev, st, hn, n, f, _ = hvar_run(sys, 4, time0, tstop, h, tol, rcen, central, max_steps)
    return ev, st, hn, n, f


def hy_run(sys, time0, h, nsteps, tol=1e-12, rcen=0.005, central=True):
    """mal_hcon's HYBRID loop (mdt_hy) on sys's democratic-heliocentric state (in place).

    Uses sys.rcrit. Returns (events, step of each event, force calls, encounter pairs)."""
    s = sys
    counters = (C.c_longlong * 2)()
    handle = lib().oracle_hy_run(s.n, s.nbig, _p(s.m), _p(s.x), _p(s.v), _p(s.ngf), s.ngflag, _p(s.jcen),
                                 _p(s.rce), _p(s.rphys), _p(s.rcrit), time0, h, int(nsteps), tol, rcen,
                                 int(central), counters)
    try:
        if lib().oracle_run_status(handle):
            raise RuntimeError("oracle HYBRID run failed")
        count = lib().oracle_run_event_count(handle)
        events = np.zeros(count, dtype=EVENT_DTYPE)
        steps = np.zeros(count, dtype=np.int32)
        lib().oracle_run_events(handle, events.ctypes.data_as(C.c_void_p), steps.ctypes.data_as(C.c_void_p))
    finally:
        lib().oracle_run_free(handle)
    return events, steps, counters[0], counters[1]


def mce_snif(h, nbig, x0, v0, x1, v1, rcrit, cap=100000):
    x0, v0, x1, v1, rcrit = map(_f64, (x0, v0, x1, v1, rcrit))
    n = len(rcrit)
    ice = np.zeros(cap, dtype=np.int32)
    jce = np.zeros(cap, dtype=np.int32)
    PI_ = C.POINTER(I)
    k = lib().oracle_mce_snif(h, n, nbig, _p(x0), _p(v0), _p(x1), _p(v1), _p(rcrit),
                              ice.ctypes.data_as(PI_), jce.ctypes.data_as(PI_), cap)
    return ice[:min(k, cap)], jce[:min(k, cap)]


def mfo_hy(sys):
    a = np.zeros((sys.n, 3))
    lib().oracle_mfo_hy(sys.n, sys.nbig, _p(sys.m), _p(sys.x), _p(sys.rcrit), _p(sys.jcen), _p(a))
    return a


def mvs_jacobian(sys, h, nsteps):
    """nsteps of mdt_mvs on sys (in place) with forward-mode derivatives of
    every test particle's final (x, v) with respect to its initial (x, v) and
    its Yarkovsky coefficient: returns J of shape (n - nbig, 6, 7)."""
    s = sys
    jac = np.zeros((s.n - s.nbig, 6, 7))
    rc = lib().oracle_mvs_jacobian(s.n, s.nbig, _p(s.m), _p(s.x), _p(s.v), _p(s.ngf), s.ngflag, _p(s.jcen), h,
                                   int(nsteps), _p(jac))
    if rc:
        raise RuntimeError("oracle Jacobian run failed")
    return jac


def hy_jacobian(sys, h, nsteps, tol=1e-12):
    """nsteps of mdt_hy on sys's democratic-heliocentric state (in place, no
    oblateness) with forward-mode derivatives of every test particle's final
    (x, v) with respect to its initial (x, v) and its Yarkovsky coefficient,
    through the encounter subsystem's BS2 substeps where it is a member: J of
    shape (n - nbig, 6, 7). Uses sys.rcrit."""
    s = sys
    jac = np.zeros((s.n - s.nbig, 6, 7))
    rc = lib().oracle_hy_jacobian(s.n, s.nbig, _p(s.m), _p(s.x), _p(s.v), _p(s.ngf), s.ngflag, _p(s.rcrit), h,
                                  int(nsteps), tol, _p(jac))
    if rc:
        raise RuntimeError("oracle HYBRID Jacobian run failed")
    return jac


def mxx_ejec(x, rmax, i0=2):
    """mxx_ejec's test (mercury6_2.for:7071-7082) on heliocentric x (n, 3):
    ascending 1-based ids of bodies j >= i0 beyond rmax."""
    x = _f64(x)
    n = len(x)
    ids = np.zeros(max(1, n), dtype=np.int32)
    k = lib().oracle_mxx_ejec(n, int(i0), _p(x), float(rmax), ids.ctypes.data_as(C.POINTER(I)))
    return ids[:k].copy()


def mio_ce(events, mcen, rcen, rmax):
    """mio_ce's 70-character record bodies (mercury6_2.for:5456-5510) of the
    close encounters (kind bit 1) among `events` (EVENT_DTYPE), in order:
    uint8 array (count, 70)."""
    ev = np.ascontiguousarray(events, dtype=EVENT_DTYPE)
    lines = np.zeros((max(1, len(ev)), 70), dtype=np.uint8)
    k = lib().oracle_mio_ce(ev.ctypes.data_as(C.c_void_p), len(ev), float(mcen), float(rcen), float(rmax),
                            lines.ctypes.data_as(C.c_void_p))
    return lines[:k].copy()


def epoch_order(epochs, tstart):
    """mxx_sync's order of the Small bodies (mxx_sort, then furthest from tstart first)."""
    e = _f64(epochs)
    order = np.zeros(max(1, len(e)), dtype=np.int32)
    lib().oracle_epoch_order(len(e), _p(e), float(tstart), order.ctypes.data_as(C.POINTER(I)))
    return order[:len(e)].copy()


def mxx_sync(sys, epoch, time, h0, tol, dtout):
    """mxx_sync's integration on sys (bodies already in its order, in place):
    returns (final time, BS steps)."""
    s = sys
    t = D(float(time))
    steps = I(0)
    ep = _f64(epoch)
    rc = lib().oracle_mxx_sync(s.n, s.nbig, _p(s.m), _p(s.x), _p(s.v), _p(s.ngf), s.ngflag, int(s.pn), _p(s.jcen),
                               _p(ep), C.byref(t), float(h0), float(tol), float(dtout), C.byref(steps))
    if rc:
        raise RuntimeError("oracle mxx_sync failed")
    return t.value, steps.value


def mxx_en(m, x, v, jcen, spin=None):
    """mxx_en (mercury6_2.for:7226-7315) of heliocentric x, v (n, 3): (e, l2)."""
    m = np.ascontiguousarray(m, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    jcen = np.ascontiguousarray(jcen, dtype=np.float64)
    sp = None if spin is None else np.ascontiguousarray(spin, dtype=np.float64)
    out = np.zeros(2)
    lib().oracle_mxx_en(len(m), _p(m), _p(x), _p(v), sp.ctypes.data_as(C.c_void_p) if sp is not None else None,
                        _p(jcen), _p(out))
    return float(out[0]), float(out[1])
