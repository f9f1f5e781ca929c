"""mdt_bs1 (BS) and mdt_bs2 (BS2) through the drop-in C ABI on the GPU against
the oracle, restating the reference's tests/test_gpu_algorithms.py:102-110
(BS2 with and without semi-active bodies, BS with semi-active bodies, 1PN,
Yarkovsky and radiation pressure, both directions). The device computes the
same statements in the same order, so states, step sizes, force counts and
rejections are compared exactly."""
import math

import numpy as np
import pytest

from adaptive_cases import compare_events, hvar_system, oracle_intervals, run_intervals
from mercuda_b200.backend import Backend
from mercuda_b200.system import K2, System, make_system

pytestmark = pytest.mark.gpu


def run_both(cuda_lib, oracle, name, sys, stop, interval=7.3, h=0.5, tol=1e-12):
    alg = {"BS": 2, "BS2": 3}[name]
    ref = sys.copy()
    be = Backend(name, cuda_lib)
    be.configure()
    be.upload(sys)
    ev, hn = run_intervals(be, sys, 0.0, stop, interval, math.copysign(h, stop), tol)
    x, v = be.download()
    forces, rejected = be.forces, be.rejected
    be.free()
    want = oracle_intervals(oracle, ref, alg, 0.0, stop, interval, math.copysign(h, stop), tol)
    return (ev, hn, x, v, forces, rejected), (want, ref)


def assert_same(got, want):
    (ev, hn, x, v, forces, rejected), ((want_ev, want_h, _, want_forces, want_rej), ref) = got, want
    assert (forces, rejected) == (want_forces, want_rej)
    assert hn == want_h
    assert np.array_equal(x, ref.x) and np.array_equal(v, ref.v), (
        np.max(np.abs(x - ref.x)), np.max(np.abs(v - ref.v)))
    compare_events(ev, want_ev)


@pytest.mark.parametrize("direction", [-1, 1])
def test_bs_semi_active(cuda_lib, oracle, direction):
    assert_same(*run_both(cuda_lib, oracle, "BS", hvar_system(massive=True, pn=1), direction * 32.0))


@pytest.mark.parametrize("massive", [False, True])
@pytest.mark.parametrize("direction", [-1, 1])
def test_bs2(cuda_lib, oracle, massive, direction):
    assert_same(*run_both(cuda_lib, oracle, "BS2", hvar_system(massive=massive, pn=0), direction * 32.0))


@pytest.mark.parametrize("name", ["BS", "BS2"])
def test_bs_halves_a_long_first_step(cuda_lib, oracle, name):
    """A 200-day first step fails every level and is halved until one passes."""
    vc = math.sqrt(K2)
    sys = System(m=np.array([K2, 1e-3 * K2, 0.0]), x=np.array([[0, 0, 0], [5.2, 0, 0], [1.0, 0, 0]]),
                 v=np.array([[0, 0, 0], [0, math.sqrt(K2 * 1.001 / 5.2), 0], [0, vc, 0]]), nbig=2)
    got, want = run_both(cuda_lib, oracle, name, sys, 400.0, interval=400.0, h=200.0)
    assert got[5] >= 1
    assert_same(got, want)


@pytest.mark.parametrize("name", ["BS", "BS2"])
def test_bs_particles_and_events(cuda_lib, oracle, name):
    """Massless particles in slots, encounters and impacts with the planets."""
    sys = make_system(seed=8, n_particles=1500, nplanets=6, near_fraction=0.05, h=4.0)
    if name == "BS":
        rng = np.random.default_rng(4)
        npart = sys.n - sys.nbig
        sys.ngf[sys.nbig:, 3] = rng.uniform(0.01, 0.3, npart)
        sys.ngf[sys.nbig:, 4] = np.exp(rng.uniform(np.log(1e-15), np.log(1e-13), npart)) * rng.choice([-1, 1], npart)
        sys.pn = 1
    got, want = run_both(cuda_lib, oracle, name, sys, 20.0, interval=20.0, h=2.0)
    assert len(want[0][0]) > 0
    assert_same(got, want)
