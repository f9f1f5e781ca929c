"""Planetary systems for the test-particle path: container, seeded synthetic
workloads and the host-side encounter limits.

Arrays keep the reference host's layout (mercury_gpu.f90:139-151): masses in
K2 units (``m = mass_in_msun * K2``, mercury6_2.for:6271), ``x``/``v`` as (n, 3)
heliocentric rows (byte-identical to Fortran x(3,n)), ``ngf`` as (n, 5) rows of
A1, A2, A3, beta, yar. Index 0 is the central body, 1..nbig-1 the Big bodies,
nbig..n-1 the Small bodies (test particles).

The workloads are seeded synthetic stand-ins with the shapes and element
distributions of the five benchmark configurations of this path; every
implementation is handed the same float64 arrays.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace

import numpy as np

K2 = 2.959122082855911e-4          # mercury.inc: Gaussian constant squared
AU_CM = 1.495978707e13             # mercury.inc: AU in cm
MSUN_G = 1.9884158605722262e33     # mercury.inc: solar mass in g
RHOCGS = AU_CM * AU_CM * AU_CM * K2 / MSUN_G   # mercury6_2.for:1364, 1 g/cm^3
DEG = np.pi / 180.0


@dataclass
class System:
    """One heliocentric planetary system (central body + Big + Small bodies)."""

    m: np.ndarray
    x: np.ndarray
    v: np.ndarray
    nbig: int
    ngf: np.ndarray | None = None
    jcen: np.ndarray = field(default_factory=lambda: np.zeros(3))
    rce: np.ndarray | None = None
    rphys: np.ndarray | None = None
    rcrit: np.ndarray | None = None
    rceh: np.ndarray | None = None
    rho: np.ndarray | None = None
    pn: int = 0

    def __post_init__(self):
        n = len(self.m)
        self.m = np.ascontiguousarray(self.m, dtype=np.float64)
        self.x = np.ascontiguousarray(np.reshape(self.x, (n, 3)), dtype=np.float64)
        self.v = np.ascontiguousarray(np.reshape(self.v, (n, 3)), dtype=np.float64)
        self.ngf = (np.zeros((n, 5)) if self.ngf is None
                    else np.ascontiguousarray(np.reshape(self.ngf, (n, 5)), dtype=np.float64))
        self.jcen = np.ascontiguousarray(self.jcen, dtype=np.float64)
        for name in ("rce", "rphys", "rcrit"):
            val = getattr(self, name)
            setattr(self, name, np.zeros(n) if val is None else np.ascontiguousarray(val, dtype=np.float64))
        self.rceh = np.ones(n) if self.rceh is None else np.asarray(self.rceh, dtype=np.float64)
        self.rho = np.full(n, RHOCGS) if self.rho is None else np.asarray(self.rho, dtype=np.float64)

    @property
    def n(self) -> int:
        return len(self.m)

    @property
    def ngflag(self) -> int:
        """Derived as in mio_in (mercury6_2.for:6360-6371): 1 = A1..A3/yar, 2 = beta, 3 = both."""
        g = self.ngf
        flag = 0
        if not g.reshape(-1).any():   # one contiguous pass: the usual all-zero case
            return flag
        if np.any(g[:, [0, 1, 2, 4]] != 0):
            flag |= 1
        if np.any(g[:, 3] != 0):
            flag |= 2
        return flag

    def copy(self) -> "System":
        return replace(self, m=self.m.copy(), x=self.x.copy(), v=self.v.copy(), ngf=self.ngf.copy(),
                       jcen=self.jcen.copy(), rce=self.rce.copy(), rphys=self.rphys.copy(),
                       rcrit=self.rcrit.copy(), rceh=self.rceh.copy(), rho=self.rho.copy())


def kepler_solve(M: np.ndarray, e: np.ndarray) -> np.ndarray:
    """Eccentric anomaly E of elliptic Kepler's equation E - e sin E = M (Newton)."""
    E = M + e * np.sin(M) * (1.0 + e * np.cos(M))
    for _ in range(50):
        f = E - e * np.sin(E) - M
        E = E - f / (1.0 - e * np.cos(E))
    return E


def elements_to_cartesian(gm, a, e, inc, node, peri, M):
    """Heliocentric position/velocity of elliptic orbits from classical elements."""
    gm, a, e, inc, node, peri, M = map(np.asarray, (gm, a, e, inc, node, peri, M))
    E = kepler_solve(np.mod(M, 2 * np.pi), e)
    cE, sE = np.cos(E), np.sin(E)
    b = a * np.sqrt(1.0 - e * e)
    px, py = a * (cE - e), b * sE                      # in the orbital plane
    nmot = np.sqrt(gm / a ** 3)
    rdot = nmot * a / (1.0 - e * cE)
    vx, vy = -a * sE * rdot / a * 1.0, b * cE * rdot / a
    cw, sw = np.cos(peri), np.sin(peri)
    cn, sn = np.cos(node), np.sin(node)
    ci, si = np.cos(inc), np.sin(inc)
    r11 = cn * cw - sn * sw * ci
    r12 = -cn * sw - sn * cw * ci
    r21 = sn * cw + cn * sw * ci
    r22 = -sn * sw + cn * cw * ci
    r31 = sw * si
    r32 = cw * si
    x = np.stack([r11 * px + r12 * py, r21 * px + r22 * py, r31 * px + r32 * py], axis=-1)
    v = np.stack([r11 * vx + r12 * vy, r21 * vx + r22 * vy, r31 * vx + r32 * vy], axis=-1)
    return x, v


def mce_init(sys: System, h: float, cefac: float = 3.0) -> System:
    """Encounter limits rce, physical radii rphys and changeover radii rcrit.

    Follows mce_init/mce_hill (mercury6_2.for:1285-1418): hill = a (m/3m1)^(1/3)
    (a -> r for unbound orbits), rce = hill * rceh, rphys = hill/a (2.25 m1/(pi rho))^(1/3),
    rcrit = max(hill * cefac, 0.4 |h| sqrt(m1/amin)). This is host-side set-up
    that the Fortran driver performs before uploading.
    """
    m, x, v = sys.m, sys.x, sys.v
    n = sys.n
    hill = np.zeros(n)
    a = np.zeros(n)
    third = 0.3333333333333333
    gm = m[0] + m[1:]
    r = np.sqrt(x[1:, 0] * x[1:, 0] + x[1:, 1] * x[1:, 1] + x[1:, 2] * x[1:, 2])
    v2 = v[1:, 0] * v[1:, 0] + v[1:, 1] * v[1:, 1] + v[1:, 2] * v[1:, 2]
    with np.errstate(divide="ignore", invalid="ignore"):
        aa = np.where(2.0 * gm == r * v2, 0.0, gm * r / (2.0 * gm - r * v2))
    aa = np.where(aa <= 0.0, r, aa)
    a[1:] = aa
    # x**(1/3) as the Fortran's real power computes it: the C library's pow,
    # one body at a time, wherever the bits matter (numpy's vectorised power
    # may differ in the last bit). For massless bodies hill = a * 0**(1/3) = 0
    # and rphys = 0 * (...), which no rounding of the power changes.
    cbrt_c = lambda q: np.array([math.pow(float(t), third) for t in q]) if len(q) else np.zeros(0)
    massive = np.nonzero(m[1:] != 0.0)[0] + 1
    with np.errstate(over="ignore", invalid="ignore"):
        hill[1:] = aa * np.power(third * m[1:] / m[0], third)
    hill[massive] = aa[massive - 1] * cbrt_c(third * m[massive] / m[0])
    temp = 2.25 * m[0] / np.pi
    sys.rce = np.zeros(n)
    sys.rphys = np.zeros(n)
    sys.rce[1:] = hill[1:] * sys.rceh[1:]
    with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
        sys.rphys[1:] = hill[1:] / a[1:] * np.power(temp / sys.rho[1:], third)
    sys.rphys[massive] = hill[massive] / a[massive] * cbrt_c(temp / sys.rho[massive])
    amin = min(9.9e29, float(np.min(a[1:]))) if n > 1 else 9.9e29
    vmax = np.sqrt(m[0] / amin)
    tmp = 0.4 * abs(h) * vmax
    sys.rcrit = np.zeros(n)
    sys.rcrit[1:] = np.maximum(hill[1:] * cefac, tmp)
    return sys


def _log_uniform(rng, lo, hi, size):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size))


def planets(rng: np.random.Generator, nplanets: int = 8, mmin: float = 1.7e-7, mmax: float = 1e-3,
            amin: float = 0.39, amax: float = 30.0, emax: float = 0.05, imax_deg: float = 3.0):
    """Big bodies: masses log-uniform [mmin, mmax] Msun, a log-spaced [amin, amax] AU."""
    mass = _log_uniform(rng, mmin, mmax, nplanets)
    a = np.exp(np.linspace(np.log(amin), np.log(amax), nplanets)) if nplanets > 1 else np.array([amin])
    e = rng.uniform(0.0, emax, nplanets)
    inc = rng.uniform(0.0, imax_deg * DEG, nplanets)
    node, peri, M = (rng.uniform(0.0, 2 * np.pi, nplanets) for _ in range(3))
    return mass, a, e, inc, node, peri, M


def make_system(seed: int = 1, n_particles: int = 10_000, nplanets: int = 8, near_fraction: float = 0.0,
                h: float = 8.0, rceh_big: float = 3.0, cefac: float = 3.0, pa=(0.5, 5.0),
                pe_max: float = 0.2, pi_max_deg: float = 10.0, planet_kw: dict | None = None,
                particle_seed=None) -> System:
    """Seeded synthetic system with the element distributions of the MVS workloads.

    Central mass 1 Msun; ``nplanets`` Big bodies (masses log-uniform 1.7e-7 to
    1e-3 Msun, a log-spaced 0.39 to 30 AU, e U[0,0.05], i U[0,3 deg]); massless
    test particles with a U[0.5,5] AU, e U[0,0.2], i U[0,10 deg]; all angles
    uniform. ``near_fraction`` of the particles are instead placed inside 5 Hill
    radii of a randomly chosen planet (a offset <= 5 R_H, same mean anomaly
    within R_H/a) so that encounter events fire. ``rceh_big`` is the Big bodies'
    ``r=`` token (encounter radius in Hill radii). With ``particle_seed`` the
    particles come from their own generator of that seed and the planets from
    ``seed`` alone: shards of one system with the same planets.
    """
    rng = np.random.default_rng(seed)
    m0 = K2
    mass, pa_, pe_, pi_, pn_, pw_, pM_ = planets(rng, nplanets, **(planet_kw or {}))
    if particle_seed is not None:
        rng = np.random.default_rng(particle_seed)
    n = 1 + nplanets + n_particles
    m = np.zeros(n)
    m[0] = m0
    m[1:1 + nplanets] = mass * K2
    x = np.zeros((n, 3))
    v = np.zeros((n, 3))
    if nplanets:
        xb, vb = elements_to_cartesian(m0 + m[1:1 + nplanets], pa_, pe_, pi_, pn_, pw_, pM_)
        x[1:1 + nplanets], v[1:1 + nplanets] = xb, vb
    a = rng.uniform(pa[0], pa[1], n_particles)
    e = rng.uniform(0.0, pe_max, n_particles)
    inc = rng.uniform(0.0, pi_max_deg * DEG, n_particles)
    node, peri, M = (rng.uniform(0.0, 2 * np.pi, n_particles) for _ in range(3))
    nnear = int(round(near_fraction * n_particles)) if nplanets else 0
    if nnear:
        idx = rng.choice(n_particles, nnear, replace=False)
        host = rng.integers(0, nplanets, nnear)
        hill = pa_[host] * np.cbrt(mass[host] / 3.0)
        a[idx] = pa_[host] + rng.uniform(-5.0, 5.0, nnear) * hill
        e[idx] = pe_[host] + rng.uniform(0.0, 0.01, nnear)
        inc[idx] = pi_[host]
        node[idx] = pn_[host]
        peri[idx] = pw_[host]
        M[idx] = pM_[host] + rng.uniform(-1.0, 1.0, nnear) * hill / pa_[host]
    if n_particles:
        xs, vs = elements_to_cartesian(np.full(n_particles, m0), a, e, inc, node, peri, M)
        x[1 + nplanets:], v[1 + nplanets:] = xs, vs
    rceh = np.ones(n)
    rceh[1:1 + nplanets] = rceh_big
    sys = System(m=m, x=x, v=v, nbig=1 + nplanets, rceh=rceh)
    return mce_init(sys, h, cefac)


def make_batch(seed: int = 1, nsys: int = 4096, nmin: int = 10, nmax: int = 5000, hmin: float = 4.0,
               hmax: float = 16.0, big_max: int = 8, near_fraction: float = 0.0):
    """Seeded batch of independent systems for the batched path: per system
    1..big_max planets (uniform), log-uniform particle count in [nmin, nmax],
    step h uniform in [hmin, hmax] days, the single-system distributions
    otherwise. Returns (systems, h)."""
    rng = np.random.default_rng(seed)
    nbig = rng.integers(1, big_max + 1, nsys)
    npart = np.exp(rng.uniform(np.log(nmin), np.log(nmax), nsys)).astype(int)
    h = rng.uniform(hmin, hmax, nsys)
    systems = [make_system(seed=int(rng.integers(1 << 30)), n_particles=int(npart[k]), nplanets=int(nbig[k]),
                           near_fraction=near_fraction, h=float(h[k]))
               for k in range(nsys)]
    return systems, h
