"""Independent high-precision two-body propagation for oracle known-answer
tests: universal-variable Kepler equation solved by bisection in 50-digit
arithmetic (mpmath), valid for elliptic, parabolic and hyperbolic orbits."""
import mpmath as mp
import numpy as np


def _stumpff(z):
    if abs(z) < mp.mpf("1e-40"):
        return mp.mpf(1) / 2, mp.mpf(1) / 6
    if z > 0:
        q = mp.sqrt(z)
        return (1 - mp.cos(q)) / z, (q - mp.sin(q)) / q ** 3
    q = mp.sqrt(-z)
    return (mp.cosh(q) - 1) / (-z), (mp.sinh(q) - q) / q ** 3


def propagate(xv, t, mu, dps=50):
    with mp.workdps(dps):
        r0 = [mp.mpf(float(c)) for c in xv[:3]]
        v0 = [mp.mpf(float(c)) for c in xv[3:]]
        mu = mp.mpf(mu)
        t = mp.mpf(t)
        rad = mp.sqrt(sum(c * c for c in r0))
        rv = sum(a * b for a, b in zip(r0, v0))
        alpha = 2 / rad - sum(c * c for c in v0) / mu
        sq = mp.sqrt(mu)

        def kepler(chi):
            c, s = _stumpff(alpha * chi * chi)
            return rv / sq * chi * chi * c + (1 - alpha * rad) * chi ** 3 * s + rad * chi - sq * t

        lo, hi = -abs(sq * t / rad) - 1, abs(sq * t / rad) + 1
        while kepler(lo) * kepler(hi) > 0:
            lo, hi = 2 * lo, 2 * hi
        for _ in range(400):
            mid = (lo + hi) / 2
            if kepler(lo) * kepler(mid) <= 0:
                hi = mid
            else:
                lo = mid
        chi = (lo + hi) / 2
        c, s = _stumpff(alpha * chi * chi)
        f = 1 - chi * chi * c / rad
        g = t - chi ** 3 * s / sq
        r = [f * a + g * b for a, b in zip(r0, v0)]
        rn = mp.sqrt(sum(q * q for q in r))
        fd = sq / (rad * rn) * (alpha * chi ** 3 * s - chi)
        gd = 1 - chi * chi * c / rn
        v = [fd * a + gd * b for a, b in zip(r0, v0)]
        return np.array([float(q) for q in r + v])
