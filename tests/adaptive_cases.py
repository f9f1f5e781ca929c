"""Shared cases of the adaptive-integrator GPU tests (BS, BS2, RADAU): the
systems of the reference's tests/test_gpu_algorithms.py:15-33 (three planets,
33 Small bodies on planar orbits, every third one semi-active on request),
mal_hvar-style interval loops on the device and on the oracle, and the event
comparison."""
import math

import numpy as np

from mercuda_b200.system import K2, System

ALGORITHMS = {"BS": 2, "BS2": 3, "RADAU": 4}


def planar_body(mass, a, e, phase):
    """Pericentre at angle `phase` in the x-y plane (m in Msun)."""
    r = a * (1 - e)
    speed = math.sqrt(K2 * (1 + e) / r)
    c, s = math.cos(phase), math.sin(phase)
    return mass * K2, [r * c, r * s, 0.0], [-speed * s, speed * c, 0.0]


def hvar_system(massive, pn, count=33):
    bigs = [planar_body(3e-6, 1.0, 0.016, 0.0), planar_body(0.001, 5.2, 0.04, 0.0),
            planar_body(0.0003, 9.5, 0.05, 0.0)]
    smalls = [planar_body(1e-8 if massive and j % 3 == 0 else 0.0, 1.6 + j * 0.012, 0.12, j * 0.37)
              for j in range(count)]
    bodies = [(K2, [0.0] * 3, [0.0] * 3)] + bigs + smalls
    m = np.array([b[0] for b in bodies])
    x = np.array([b[1] for b in bodies])
    v = np.array([b[2] for b in bodies])
    n = len(m)
    ngf = np.zeros((n, 5))
    if pn:
        ngf[4:, 4] = 1e-12
        ngf[4:, 3] = 0.001
    rce = np.full(n, 0.05)
    rphys = np.full(n, 1e-4)
    return System(m=m, x=x, v=v, nbig=4, ngf=ngf, rce=rce, rphys=rphys, pn=int(pn))


def run_intervals(be, sys, start, stop, interval, h, tol, rcen=0.005, update_limits=False):
    """Output-interval loop around mal_hvar's: one hvar_run per interval."""
    direction = math.copysign(1.0, stop - start)
    t = start
    events = []
    while abs(stop - t) > 0:
        tout = t + direction * min(interval, abs(stop - t))
        ev, _, h, _ = be.hvar_run(t, tout, h, tol, rcen)
        events.append(ev)
        t = tout
        if update_limits:
            be.limits(sys.rce)
    return np.concatenate(events) if events else events, h


def oracle_intervals(oracle, sys, algorithm, start, stop, interval, h, tol, rcen=0.005):
    """Returns (events, h, steps, forces, rejected)."""
    direction = math.copysign(1.0, stop - start)
    t = start
    events = []
    steps = forces = rejected = 0
    while abs(stop - t) > 0:
        tout = t + direction * min(interval, abs(stop - t))
        ev, _, h, s, f, r = oracle.hvar_run(sys, algorithm, t, tout, h, tol, rcen)
        events.append(ev)
        steps += s
        forces += f
        rejected += r
        t = tout
    return np.concatenate(events), h, steps, forces, rejected


def compare_events(got, want):
    key = lambda e: (min(e["i"], e["j"]), max(e["i"], e["j"]), e["kind"], round(float(e["time"]), 6))
    g = sorted(got, key=key)
    w = sorted(want, key=key)
    assert len(g) == len(w)
    for a, b in zip(g, w):
        assert (a["i"], a["j"], a["kind"], a["now"]) == (b["i"], b["j"], b["kind"], b["now"])
        assert abs(a["time"] - b["time"]) <= 1e-9 * max(1.0, abs(b["time"]))
        if a["kind"] != 8:
            assert np.array_equal(a["xi"], b["xi"]) and np.array_equal(a["xj"], b["xj"])
