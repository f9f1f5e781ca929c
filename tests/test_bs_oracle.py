"""Known answers for the oracle's adaptive integrators mdt_bs1 (BS), mdt_bs2
(BS2) and mdt_ra15 (RADAU): the reference's exact-parabola check for every
method (tests/test_validation_guards.py:112-125, GM = 1 so the zero-energy
orbit is exact in binary64) and exact circular orbits in both directions
(tests/test_release.py:35-48)."""
import math

import numpy as np
import pytest

from mercuda_b200.system import K2, System

ALGORITHMS = {"BS": 2, "BS2": 3, "RADAU": 4}


@pytest.mark.parametrize("name", list(ALGORITHMS))
def test_exact_parabola(oracle, name):
    s = System(m=np.array([1.0, 0.0]), x=np.array([[0, 0, 0], [0.5, 0, 0]]),
               v=np.array([[0, 0, 0], [0, 2.0, 0]]), nbig=1)
    oracle.hvar_run(s, ALGORITHMS[name], 0.0, 0.125, 0.125 / 16, 1e-13, central=False)
    mean = 2 * 0.125
    d = mean
    for _ in range(12):
        d -= (d + d ** 3 / 3 - mean) / (1 + d * d)
    speed = 2 / (1 + d * d)
    truth = np.array([0.5 * (1 - d * d), d, 0, -d * speed, speed, 0])
    got = np.concatenate([s.x[1], s.v[1]])
    assert np.max(np.abs(got - truth)) < 1e-11


@pytest.mark.parametrize("name,bound", [("BS", 1e-11), ("BS2", 1e-11), ("RADAU", 1e-12)])
@pytest.mark.parametrize("sign", [-1, 1])
def test_circular_orbit_1000_days(oracle, name, bound, sign):
    vc = math.sqrt(K2)
    s = System(m=np.array([K2, 0.0]), x=np.array([[0, 0, 0], [1.0, 0, 0]]),
               v=np.array([[0, 0, 0], [0, vc, 0]]), nbig=1)
    _, _, _, steps, forces, rejected = oracle.hvar_run(s, ALGORITHMS[name], 0.0, sign * 1000.0, sign * 1.0, 1e-12,
                                                       central=False)
    th = vc * 1000.0 * sign
    assert np.max(np.abs(s.x[1] - [math.cos(th), math.sin(th), 0.0])) < bound
    assert np.max(np.abs(s.v[1] / vc - [-math.sin(th), math.cos(th), 0.0])) < 10 * bound
    assert steps > 10 and forces > steps


def test_bs_halves_a_step_that_is_too_long(oracle):
    """A 200-day first step on a 1 AU orbit fails the tolerance at every level:
    mdt_bs1/mdt_bs2 halve it (rejected_steps) until a level passes."""
    for alg in (2, 3):
        vc = math.sqrt(K2)
        s = System(m=np.array([K2, 0.0]), x=np.array([[0, 0, 0], [1.0, 0, 0]]),
                   v=np.array([[0, 0, 0], [0, vc, 0]]), nbig=1)
        _, _, _, steps, _, rejected = oracle.hvar_run(s, alg, 0.0, 200.0, 200.0, 1e-12, central=False,
                                                      max_steps=1)
        assert steps == 1 and rejected >= 1
