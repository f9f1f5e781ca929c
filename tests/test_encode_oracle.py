"""The oracle's mio_ce record encoding checked against a second, independent
restatement written here in Python with Fortran's substring assignment
semantics (c(a:b) = s pads or truncates s to b - a + 1 characters, later
assignments overwrite earlier ones): mio_ce (mercury6_2.for:5456-5510),
mio_fl2c (5885-5918), mio_re2c (6926-6957), mco_x2ov (3057-3086). Both use the
host's libm, so the lines must agree byte for byte; plus hand-derived values
of the base-224 writer."""
import math

import numpy as np

from mercuda_b200.backend import EVENT_DTYPE

PI = 3.141592653589793
TWOPI = PI * 2.0


def re2c(x, xmin, xmax):
    y = (x - xmin) / (xmax - xmin)
    if y >= 1.0:
        return bytes([255] * 8)
    if y > 0.0:
        out, z = [], y
        for _ in range(8):
            z = math.fmod(z, 1.0) * 224.0
            out.append(int(z) + 32)
        return bytes(out)
    return b" " * 8


def powi(x, m):
    n, y = abs(m), None
    y = x if n % 2 else 1.0
    n >>= 1
    while n:
        x = x * x
        if n % 2:
            y = y * x
        n >>= 1
    return 1.0 / y if m < 0 else y


def fl2c(x):
    ex = 0
    if x == 0.0:
        y = 0.5
    else:
        ax = abs(x)
        ex = int(math.log10(ax))
        if ax >= 1.0:
            ex += 1
        y = ax * powi(10.0, -ex)
        if y == 1.0:
            y, ex = y * 0.1, ex + 1
        y = math.copysign(y, x) * 0.5 + 0.5
    s = bytearray(re2c(y, 0.0, 1.0))
    s[7] = min(223, max(0, ex + 112)) + 32
    return bytes(s)


def x2ov(rcen, rmax, mcen, q):
    x, y, z, u, v, w = q
    r = math.sqrt(x * x + y * y + z * z)
    v2 = u * u + v * v + w * w
    be = (mcen + 0.0) / r
    temp = (0.5 * v2) / be
    return (math.log10(min(max(r, rcen), rmax) / rcen),
            math.fmod(math.acos(z / r) + TWOPI, TWOPI), math.fmod(math.atan2(y, x) + TWOPI, TWOPI),
            1.0 / (1.0 + 2.0 * temp * temp),
            math.fmod(math.acos(w / math.sqrt(v2)) + TWOPI, TWOPI), math.fmod(math.atan2(v, u) + TWOPI, TWOPI))


def record(e, mcen, rcen, rmax):
    c = bytearray(b" " * 80)

    def put(a, b, s):
        c[a - 1:b] = (s + b" " * 12)[:b - a + 1]

    rfac = math.log10(rmax / rcen)
    put(1, 8, fl2c(float(e["time"])))
    put(9, 16, re2c(float(e["i"] - 1), 0.0, 11239423.99))
    put(12, 19, re2c(float(e["j"] - 1), 0.0, 11239423.99))
    put(15, 22, fl2c(float(e["distance"])))
    for q, o, wide in ((e["xi"], 23, 0), (e["xj"], 47, 4)):
        fr, th, ph, fv, vth, vph = x2ov(rcen, rmax, mcen, [float(t) for t in q])
        put(o, o + 7, re2c(fr, 0.0, rfac))
        put(o + 4, o + 11, re2c(th, 0.0, PI))
        put(o + 8, o + 15, re2c(ph, 0.0, TWOPI))
        put(o + 12, o + 19, re2c(fv, 0.0, 1.0))
        put(o + 16, o + 23 + wide, re2c(vth, 0.0, PI))
        put(o + 20, o + 27 + wide, re2c(vph, 0.0, TWOPI))
    return bytes(c[:70])


def test_base224_writer_known_values():
    assert re2c(0.5, 0.0, 1.0) == bytes([144] + [32] * 7)
    assert re2c(1.0, 0.0, 1.0) == bytes([255] * 8) and re2c(0.0, 0.0, 1.0) == b" " * 8
    assert fl2c(1.0)[7] == 113 + 32 and fl2c(0.0) == bytes([144] + [32] * 6 + [112 + 32])


def test_oracle_mio_ce_matches_second_restatement(oracle):
    rng = np.random.default_rng(11)
    n = 500
    ev = np.zeros(n, dtype=EVENT_DTYPE)
    ev["i"] = rng.integers(1, 10, n)
    ev["j"] = rng.integers(10, 30000000, n)
    ev["kind"] = rng.choice([1, 2, 3], n)
    ev["time"] = rng.uniform(-1e5, 1e6, n)
    ev["time"][:4] = [0.0, 1000.0, 0.001, 1.0]
    ev["distance"] = np.exp(rng.uniform(np.log(1e-6), np.log(200.0), n))
    ev["xi"][:, :3] = rng.normal(0, 30, (n, 3))
    ev["xi"][:, 3:] = rng.normal(0, 0.01, (n, 3))
    ev["xj"][:, :3] = rng.normal(0, 1, (n, 3))
    ev["xj"][:, 3:] = rng.normal(0, 0.02, (n, 3))
    mcen, rcen, rmax = 2.959122082855911e-4, 0.005, 100.0
    got = oracle.mio_ce(ev, mcen, rcen, rmax)
    want = [record(e, mcen, rcen, rmax) for e in ev if e["kind"] & 1]
    assert got.shape == (len(want), 70)
    for g, w in zip(got, want):
        assert bytes(g) == w
