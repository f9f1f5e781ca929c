"""mxx_en (mercury6_2.for:7226-7315) in the oracle: known answers, and the
property the device version relies on — massless bodies add exactly zero."""
import numpy as np

from mercuda_b200.system import K2, make_system


def test_two_body_circular_orbit(oracle):
    m = np.array([K2, 1e-3 * K2])
    mu, a = m.sum(), 1.7
    x = np.array([[0.0, 0.0, 0.0], [a, 0.0, 0.0]])
    v = np.array([[0.0, 0.0, 0.0], [0.0, np.sqrt(mu / a), 0.0]])
    e, l2 = oracle.mxx_en(m, x, v, np.zeros(3))
    mred = m[0] * m[1] / mu
    assert abs(e - (-m[0] * m[1] / (2 * a))) <= 1e-15 * abs(e)
    assert abs(l2 - mred * np.sqrt(mu * a)) <= 1e-15 * l2


def test_spin_adds_to_angular_momentum(oracle):
    m = np.array([K2, 1e-3 * K2])
    x = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]])
    v = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 0.0]])
    s = np.array([[0.0, 0.0, 2.0e-9], [0.0, 0.0, 1.0e-9]])
    _, l2 = oracle.mxx_en(m, x, v, np.zeros(3), s)
    assert abs(l2 - 3.0e-9) <= 1e-15 * 3.0e-9


def test_oblateness_term(oracle):
    """Equatorial body: the J2 term is m0 m1 J2 R^2 / r^3 * (-1/2)."""
    m = np.array([K2, 1e-9 * K2])
    r = 0.01
    x = np.array([[0.0, 0.0, 0.0], [r, 0.0, 0.0]])
    v = np.zeros((2, 3))
    jcen = np.array([1e-7, 0.0, 0.0])
    e0, _ = oracle.mxx_en(m, x, v, np.zeros(3))
    e1, _ = oracle.mxx_en(m, x, v, jcen)
    want = m[0] * m[1] / r * (jcen[0] / r**2) * (-0.5)
    assert abs((e1 - e0) - want) <= 1e-9 * abs(want)


def test_massless_bodies_add_exactly_zero(oracle):
    s = make_system(seed=4, n_particles=500)
    full = oracle.mxx_en(s.m, s.x, s.v, s.jcen)
    big = oracle.mxx_en(s.m[:s.nbig], s.x[:s.nbig], s.v[:s.nbig], s.jcen)
    assert full == big
    jc = np.array([1e-8, -2e-12, 3e-16])
    assert oracle.mxx_en(s.m, s.x, s.v, jc) == oracle.mxx_en(s.m[:s.nbig], s.x[:s.nbig], s.v[:s.nbig], jc)
