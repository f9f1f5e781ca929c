"""Known answers of the force laws (the reference's own unit tests,
tests/test_mercury.py:18-111, restated against the oracle) and a RADAU
circular-orbit check (tests/test_release.py:35-48)."""
import math

import numpy as np

from mercuda_b200.system import K2, System

LIGHT = 299792458 * 86400 / 149597870700
SW = 0.3


def test_pr_vector_law_and_rotation_invariance(oracle):
    rng = np.random.default_rng(7)
    n = 64
    m = np.array([K2] + [0.0 if i % 2 else 1e-9 for i in range(n - 1)])
    x = np.vstack([[0, 0, 0], rng.uniform(-4, 4, (n - 1, 3))])
    v = np.vstack([[0, 0, 0], rng.uniform(-0.1, 0.1, (n - 1, 3))])
    ngf = np.zeros((n, 5))
    ngf[1:, 3] = rng.uniform(1e-4, 0.5, n - 1)
    a = oracle.force_term("pr", m, x, v, ngf)
    for j in range(1, n):
        if m[j]:
            assert np.all(a[j] == 0)
            continue
        r = np.linalg.norm(x[j])
        vr = x[j] @ v[j] / r
        f = K2 * ngf[j, 3] / r ** 2
        want = f * ((1 - (1 + SW) * vr / LIGHT) * x[j] / r - (1 + SW) * v[j] / LIGHT)
        assert np.max(np.abs(a[j] - want)) < 1e-14 * np.max(np.abs(want))
    ang = [0.7, -1.3, 2.1]

    def rot(c):
        c = np.array(c, dtype=float)
        for axis, t in enumerate(ang):
            i, k = [q for q in range(3) if q != axis]
            ct, st = math.cos(t), math.sin(t)
            c[..., i], c[..., k] = ct * c[..., i] - st * c[..., k], st * c[..., i] + ct * c[..., k]
        return c

    ra = oracle.force_term("pr", m, rot(x), rot(v), ngf)
    want = rot(a)
    for j in range(1, n):
        scale = np.max(np.abs(want[j])) or 1.0
        assert np.max(np.abs(ra[j] - want[j])) < 1e-13 * scale


def test_pn_analytic_and_reversal(oracle):
    x = np.array([[0, 0, 0], [.4, .3, .1]])
    v = np.array([[0, 0, 0], [-.01, .025, .003]])
    m = np.array([K2, 0.0])
    a = oracle.force_term("pn", m, x, v, np.zeros((2, 5)))
    r = np.linalg.norm(x[1]); rv = x[1] @ v[1]; v2 = v[1] @ v[1]
    want = K2 / (LIGHT ** 2 * r ** 3) * ((4 * K2 / r - v2) * x[1] + 4 * rv * v[1])
    assert np.max(np.abs(a[1] / want - 1)) < 1e-14
    a2 = oracle.force_term("pn", m, x, -v, np.zeros((2, 5)))
    assert np.array_equal(a, a2)


def test_yar_inverse_square_and_direction(oracle):
    for r in [1.0, 2.0, 20.0]:
        for sign in [-1, 1]:
            yar = sign * 1e-10
            ngf = np.zeros((2, 5)); ngf[1, 4] = yar
            a = oracle.force_term("ngf", np.zeros(2), np.array([[0, 0, 0], [r, 0, 0]]),
                                  np.array([[0, 0, 0], [.01, .02, 0]]), ngf)
            assert a[1, 0] == 0.0 and a[1, 2] == 0.0
            assert abs(a[1, 1] / (yar / r ** 2) - 1) < 1e-14


def test_cometary_a2_and_yar_are_independent(oracle):
    for radius in [1.0, 2.0, 20.0]:
        for comet in [0.0, -2e-10, 2e-7]:
            for thermal in [0.0, 3e-11]:
                ngf = np.zeros((2, 5)); ngf[1, 1] = comet; ngf[1, 4] = thermal
                a = oracle.force_term("ngf", np.zeros(2), np.array([[0, 0, 0], [radius, 0, 0]]),
                                      np.array([[0, 0, 0], [.01, .02, 0]]), ngf)
                q = radius / 2.808
                g = .111262 * q ** (-2.15) * (1 + q ** 5.093) ** (-4.6142)
                want = (comet * g if radius ** 2 < 88 or abs(comet) > 1e-7 else 0) + thermal / radius ** 2
                assert abs(a[1, 1] - want) <= max(abs(want) * 2e-14, 1e-30)
                assert a[1, 0] == 0.0 and a[1, 2] == 0.0


def test_radau_circular_orbit_1000_days(oracle):
    """RADAU on a circular orbit at 1 AU for 1000 d at tol 1e-12 stays within
    1e-12 of the analytic solution (the reference's release regression)."""
    vc = math.sqrt(K2)
    s = System(m=np.array([K2, 0.0]), x=np.array([[0, 0, 0], [1.0, 0, 0]]),
               v=np.array([[0, 0, 0], [0, vc, 0]]), nbig=1)
    oracle.ra15_run(s, 0.0, 1000.0, 1.0, 1e-12, central=False)
    th = vc * 1000.0
    want = np.array([math.cos(th), math.sin(th), 0.0])
    assert np.max(np.abs(s.x[1] - want)) < 1e-12
